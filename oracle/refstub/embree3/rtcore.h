// Build-only stand-in for the Embree 3 API header.
//
// Test infrastructure: it lets the reference renderer (Native/renderer.cu and
// Native/embree.cuh) compile on a machine without the Embree SDK, so its
// host-side BVH builder, traversal, sampler and integrator can be run as the
// parity checker. Only the names Native/embree.cuh uses are declared. Nothing
// here links against or emulates Embree: Native/embree.cuh resolves the real
// library with dlopen("libembree3.so.3") at run time, which fails when Embree
// is absent, so the reference's backend 3 reports "Embree unavailable".
// The harness in oracle/ never selects backend 3.
#pragma once
#include <cstddef>

typedef struct RTCDeviceTy* RTCDevice;
typedef struct RTCSceneTy* RTCScene;
typedef struct RTCGeometryTy* RTCGeometry;

enum RTCError { RTC_ERROR_NONE = 0, RTC_ERROR_UNKNOWN = 1 };
enum RTCSceneFlags { RTC_SCENE_FLAG_NONE = 0, RTC_SCENE_FLAG_ROBUST = 4 };
enum RTCBuildQuality { RTC_BUILD_QUALITY_LOW = 0, RTC_BUILD_QUALITY_MEDIUM = 1, RTC_BUILD_QUALITY_HIGH = 2 };
enum RTCGeometryType { RTC_GEOMETRY_TYPE_TRIANGLE = 0 };
enum RTCBufferType { RTC_BUFFER_TYPE_INDEX = 0, RTC_BUFFER_TYPE_VERTEX = 1 };
enum RTCFormat { RTC_FORMAT_UINT3 = 0x5003, RTC_FORMAT_FLOAT3 = 0x9003 };
#define RTC_INVALID_GEOMETRY_ID ((unsigned)-1)

struct RTCRay {
    float org_x, org_y, org_z, tnear;
    float dir_x, dir_y, dir_z, time;
    float tfar;
    unsigned mask, id, flags;
};
struct RTCHit {
    float Ng_x, Ng_y, Ng_z;
    float u, v;
    unsigned primID, geomID, instID[1];
};
struct RTCRayHit { RTCRay ray; RTCHit hit; };
struct RTCRayN;
struct RTCHitN;
struct RTCIntersectContext { unsigned flags; void* filter; unsigned instID[1]; };
inline void rtcInitIntersectContext(RTCIntersectContext* context) {
    context->flags = 0; context->filter = nullptr; context->instID[0] = (unsigned)-1;
}

struct RTCFilterFunctionNArguments {
    int* valid;
    void* geometryUserPtr;
    const void* context;
    RTCRayN* ray;
    RTCHitN* hit;
    unsigned N;
};
typedef void (*RTCFilterFunctionN)(const RTCFilterFunctionNArguments* args);

// Field accessors over the SoA packet layout (ray/hit fields N floats apart).
inline float& rtcStubRayField(RTCRayN* ray, unsigned N, unsigned i, unsigned field) {
    return reinterpret_cast<float*>(ray)[field * N + i];
}
inline float& RTCRayN_dir_x(RTCRayN* ray, unsigned N, unsigned i) { return rtcStubRayField(ray, N, i, 4); }
inline float& RTCRayN_dir_y(RTCRayN* ray, unsigned N, unsigned i) { return rtcStubRayField(ray, N, i, 5); }
inline float& RTCRayN_dir_z(RTCRayN* ray, unsigned N, unsigned i) { return rtcStubRayField(ray, N, i, 6); }
inline float& RTCHitN_Ng_x(RTCHitN* hit, unsigned N, unsigned i) { return reinterpret_cast<float*>(hit)[0 * N + i]; }
inline float& RTCHitN_Ng_y(RTCHitN* hit, unsigned N, unsigned i) { return reinterpret_cast<float*>(hit)[1 * N + i]; }
inline float& RTCHitN_Ng_z(RTCHitN* hit, unsigned N, unsigned i) { return reinterpret_cast<float*>(hit)[2 * N + i]; }
inline unsigned& RTCHitN_primID(RTCHitN* hit, unsigned N, unsigned i) { return reinterpret_cast<unsigned*>(hit)[5 * N + i]; }

// Declarations only: Native/embree.cuh takes their types with decltype and
// binds them with dlsym. They are never defined or called here.
RTCDevice rtcNewDevice(const char* config);
RTCScene rtcNewScene(RTCDevice device);
void rtcSetSceneFlags(RTCScene scene, RTCSceneFlags flags);
void rtcSetSceneBuildQuality(RTCScene scene, RTCBuildQuality quality);
RTCGeometry rtcNewGeometry(RTCDevice device, RTCGeometryType type);
void* rtcSetNewGeometryBuffer(RTCGeometry geometry, RTCBufferType type, unsigned slot, RTCFormat format,
                              size_t byteStride, size_t itemCount);
void rtcSetGeometryUserData(RTCGeometry geometry, void* ptr);
void rtcSetGeometryIntersectFilterFunction(RTCGeometry geometry, RTCFilterFunctionN filter);
void rtcSetGeometryOccludedFilterFunction(RTCGeometry geometry, RTCFilterFunctionN filter);
void rtcCommitGeometry(RTCGeometry geometry);
unsigned rtcAttachGeometry(RTCScene scene, RTCGeometry geometry);
void rtcReleaseGeometry(RTCGeometry geometry);
void rtcCommitScene(RTCScene scene);
RTCError rtcGetDeviceError(RTCDevice device);
void rtcReleaseScene(RTCScene scene);
void rtcReleaseDevice(RTCDevice device);
void rtcIntersect1(RTCScene scene, RTCIntersectContext* context, RTCRayHit* rayhit);
void rtcOccluded1(RTCScene scene, RTCIntersectContext* context, RTCRay* ray);
