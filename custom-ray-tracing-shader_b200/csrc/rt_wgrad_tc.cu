// Weight gradient of the denoiser's 3x3 convolutions on the fifth-generation
// tensor cores: dw[tap][ci][co] += sum over pixels p of
// x[p + off(tap)][ci] * dy[p][co], with x and dy NHWC BF16 and dw FP32.
//
// Per tap this is a GEMM whose K is the pixels. Both operands are staged by
// TMA as planes of 8 channels x pixels x 16 bytes (one image row segment of
// 128 output pixels per stage: x with a one-pixel halo, dy without), which
// is the MN-major no-swizzle operand layout: core matrices of 8 pixels (K)
// x 8 channels (M or N), K groups 128 bytes apart (LBO), channel groups one
// plane apart (SBO). The horizontal tap offset is a 16-byte shift of x's
// start address, so a block handles one tap row dy and keeps the three dx
// taps in three tensor-memory accumulators over its whole range of row
// segments (split K), then adds them to dw with FP32 atomics.
//
// M is 128 rows of one operand and N the channels of the other: M = input
// channels (a block of 128 of them) when cin >= cout, else M = output
// channels; the smaller channel count is N, so the padding of M to 128 rows
// costs the least. Rows beyond the real channels read stale staging planes
// and are dropped (a row of D depends on its row of A only).
//
// Roles: warp 0 issues the TMA loads into a ring of stages, warp 1 issues
// the MMAs (24 per stage: 3 dx taps x 8 K steps of 16 pixels) and owns the
// tensor memory, warps 2-5 drain the accumulators at the end. Waits are
// bounded as in rt_conv_pipe.cu.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "rt_conv_tc.cuh"

namespace rt {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kM = 128;                 // pixels per row segment (K per stage)
constexpr int kHaloPx = kM + 2;
constexpr uint32_t kXPlane = 2176;      // 130 pixels x 16 bytes, padded to 128 bytes
constexpr uint32_t kDPlane = kM * 16;   // 2,048
constexpr int kThreads = 192;
constexpr int kMaxStages = 6;
constexpr uint32_t kHeader = 1024;

struct WgradArgs {
    int n, h, w, cin, cout;
    int tilesPerRow, segments, segPerBlock;
    int mIsX;            // 1: M = input channels (from mBase), N = output channels; 0: M = output, N = input
    int mBase;           // first input channel of the M block (M = input channels)
    int mValid, nDim;
    int xPlanes, dPlanes;          // planes loaded per stage
    uint32_t xBytes, stageBytes;   // staging of x (16 or xPlanes planes) and of a whole stage
    int stages;
    uint32_t accCols, tmemCols;
    float* dw;
    int* errorFlag;
    unsigned long long waitLimitNs;
};

struct Header {
    static constexpr uint32_t full = 0;                 // kMaxStages
    static constexpr uint32_t empty = 8 * kMaxStages;   // kMaxStages
    static constexpr uint32_t done = 16 * kMaxStages;
    static constexpr uint32_t drain = 16 * kMaxStages + 8;
    static constexpr uint32_t tmemSlot = 16 * kMaxStages + 16;
    static constexpr uint32_t abort = 16 * kMaxStages + 20;
};

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t nowNs() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void barInit(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void barExpectTx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool barTryWait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity), "r"(1000u)
        : "memory");
    return done != 0;
}
__device__ bool waitPhase(uint32_t bar, uint32_t parity, volatile int* abortFlag, uint64_t limitNs) {
    if (barTryWait(bar, parity)) return true;
    const uint64_t deadline = nowNs() + limitNs;
    for (;;) {
        if (barTryWait(bar, parity)) return true;
        if (*abortFlag) return false;
        if (nowNs() > deadline) { *abortFlag = 1; return false; }
    }
}
__device__ __forceinline__ bool waitPhaseWarp(uint32_t bar, uint32_t parity, volatile int* abortFlag,
                                              uint64_t limitNs) {
    bool ok = true;
    if ((threadIdx.x & 31) == 0) ok = waitPhase(bar, parity, abortFlag, limitNs);
    return __shfl_sync(0xFFFFFFFFu, ok ? 1 : 0, 0) != 0;
}
__device__ void pollPhase(uint32_t bar, uint32_t parity, uint64_t limitNs) {
    const uint64_t deadline = nowNs() + limitNs;
    while (!barTryWait(bar, parity) && nowNs() < deadline) {
    }
}
__device__ __forceinline__ void tmaLoad4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both MN-major
// (bits 15 and 16), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idescMnMajor(int m, int n) {
    return ummaInstrDescBf16(m, n) | (1u << 15) | (1u << 16);
}

__global__ void __launch_bounds__(kThreads) wgradTcKernel(const __grid_constant__ CUtensorMap xMap,
                                                         const __grid_constant__ CUtensorMap dMap, WgradArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = smemAddr(smem);
    volatile int* abortFlag = reinterpret_cast<volatile int*>(smem + Header::abort);
    const uint32_t stage0 = base + kHeader;
    const int S = a.stages;
    const int dy = blockIdx.y;
    const int mBase = a.mBase;
    const long long seg0 = (long long)blockIdx.x * a.segPerBlock;
    const long long seg1 = seg0 + a.segPerBlock < a.segments ? seg0 + a.segPerBlock : (long long)a.segments;
    const uint64_t limit = a.waitLimitNs;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            barInit(base + Header::full + 8 * s, 1);
            barInit(base + Header::empty + 8 * s, 1);
        }
        barInit(base + Header::done, 1);
        barInit(base + Header::drain, 1);
        *abortFlag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(base + Header::tmemSlot),
                     "r"(a.tmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + Header::tmemSlot);

    if (warp == 0) {
        // ---- producer: one stage per row segment ----
        long long k = 0;
        bool ok = true;
        for (long long s = seg0; s < seg1; s++, k++) {
            const int st = (int)(k % S);
            if (!waitPhaseWarp(base + Header::empty + 8 * st, (uint32_t)(((k / S) & 1) ^ 1), abortFlag, limit)) { ok = false; break; }
            if (lane == 0) {
                const int xt = (int)(s % a.tilesPerRow);
                const long long row = s / a.tilesPerRow;
                const int y = (int)(row % a.h), img = (int)(row / a.h), x0 = xt * kM;
                const uint32_t fb = base + Header::full + 8 * st;
                const uint32_t xs = stage0 + (uint32_t)st * a.stageBytes, ds = xs + a.xBytes;
                barExpectTx(fb, (uint32_t)a.xPlanes * kHaloPx * 16u + (uint32_t)a.dPlanes * kDPlane);
                const int xc0 = a.mIsX ? mBase : 0;
                for (int g = 0; g < a.xPlanes; g++)
                    tmaLoad4(xs + (uint32_t)g * kXPlane, &xMap, xc0 + g * 8, x0 - 1, y + dy - 1, img, fb);
                for (int g = 0; g < a.dPlanes; g++)
                    tmaLoad4(ds + (uint32_t)g * kDPlane, &dMap, g * 8, x0, y, img, fb);
            }
            __syncwarp();
        }
        if (!ok) *abortFlag = 1;
        // Every issued load lands before the block exits (latest phase of
        // each of the last S stages).
        if (lane == 0)
            for (long long e = k > S ? k - S : 0; e < k; e++)
                pollPhase(base + Header::full + 8 * (int)(e % S), (uint32_t)((e / S) & 1), limit);
        __syncwarp();
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            bool ok = true;
            const uint32_t idesc = idescMnMajor(kM, a.nDim);
            // Stage and phase as running counters; descriptors as compile-
            // time offsets from two per-stage bases (a single issuing
            // thread that computes descriptors per MMA issues several
            // times slower than the tensor pipe runs).
            long long k = 0;
            int st = 0;
            uint32_t parity = 0;
            for (long long s = seg0; s < seg1 && ok; s++, k++) {
                ok = waitPhase(base + Header::full + 8 * st, parity, abortFlag, limit);
                if (!ok) break;
                tcFenceAfter();
                const uint32_t xs = stage0 + (uint32_t)st * a.stageBytes, ds = xs + a.xBytes;
                // 16 pixels per MMA: 2 core-matrix groups of 8 along K (LBO = 128 bytes),
                // next 16 pixels 256 bytes on; tap dx one pixel (16 bytes) on.
                const uint64_t xBase = ummaSmemDesc(xs, 128u, kXPlane), dBase = ummaSmemDesc(ds, 128u, kDPlane);
                const uint32_t first = k > 0 ? 1u : 0u;
                if (a.mIsX) {
#pragma unroll
                    for (int dx = 0; dx < 3; dx++)
#pragma unroll
                        for (int kk = 0; kk < kM / 16; kk++)
                            mma(tmem + (uint32_t)dx * a.accCols, xBase + (uint64_t)(dx + 16 * kk), dBase + (uint64_t)(16 * kk),
                                idesc, (first || kk > 0) ? 1u : 0u);
                } else {
#pragma unroll
                    for (int dx = 0; dx < 3; dx++)
#pragma unroll
                        for (int kk = 0; kk < kM / 16; kk++)
                            mma(tmem + (uint32_t)dx * a.accCols, dBase + (uint64_t)(16 * kk), xBase + (uint64_t)(dx + 16 * kk),
                                idesc, (first || kk > 0) ? 1u : 0u);
                }
                commit(base + Header::empty + 8 * st);
                if (++st == S) { st = 0; parity ^= 1u; }
            }
            if (ok) {
                commit(base + Header::done);
                // The releases' arrivals land before shared memory goes away.
                for (long long e = k > S ? k - S : 0; e < k; e++)
                    pollPhase(base + Header::empty + 8 * (int)(e % S), (uint32_t)((e / S) & 1), limit);
            } else {
                *abortFlag = 1;
                commit(base + Header::drain);
                pollPhase(base + Header::drain, 0u, limit);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: add the three accumulators to dw ----
        const int quarter = warp & 3;
        const bool ok = waitPhaseWarp(base + Header::done, 0u, abortFlag, limit);
        if (ok && seg1 > seg0) {
            tcFenceAfter();
            const int r = quarter * 32 + lane;  // accumulator row of this thread
            for (int dx = 0; dx < 3; dx++) {
                const int tap = dy * 3 + dx;
                for (int c = 0; c < a.nDim; c += 16) {
                    uint32_t v[16];
                    tmemLoad16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)dx * a.accCols + (uint32_t)c, v);
                    if (r >= a.mValid) continue;
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const float f = __uint_as_float(v[j]);
                        if (f == 0.0f) continue;
                        const int ci = a.mIsX ? mBase + r : c + j;
                        const int co = a.mIsX ? c + j : r;
                        atomicAdd(a.dw + ((size_t)tap * a.cin + ci) * a.cout + co, f);
                    }
                }
            }
        }
    }
    tcFenceBefore();
    __syncthreads();
    if (threadIdx.x == 0 && *abortFlag) atomicExch(a.errorFlag, 1);
    if (warp == 1) {
        tcFenceAfter();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(a.tmemCols)
                     : "memory");
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encodeTiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

bool makeActivationMap(CUtensorMap* map, const bf16* ptr, int n, int h, int w, int c, uint32_t boxPixels) {
    auto fn = encodeTiled();
    if (!fn) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)w * c * 2, (cuuint64_t)h * w * c * 2};
    const cuuint32_t box[4] = {8, boxPixels, 1, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16*>(ptr), dims, strides, box, elem,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool wgradTcSupported(int cin, int cout) {
    const int small = std::min(cin, cout);
    return cin % 16 == 0 && cout % 16 == 0 && cin >= 16 && cout >= 16 && cout <= 128 && small <= 128 &&
           cin <= 256 && 3 * small <= 512;
}

cudaError_t wgradTc(const bf16* x, const bf16* dy, int n, int h, int w, int cin, int cout, float* dw, int* errorFlag,
                    cudaStream_t stream) {
    if (!wgradTcSupported(cin, cout) || n < 1 || h < 1 || w < 1 || !errorFlag) return cudaErrorNotSupported;
    CUtensorMap xMap{}, dMap{};
    if (!makeActivationMap(&xMap, x, n, h, w, cin, kHaloPx) || !makeActivationMap(&dMap, dy, n, h, w, cout, kM))
        return cudaErrorNotSupported;
    WgradArgs a{};
    a.n = n; a.h = h; a.w = w; a.cin = cin; a.cout = cout;
    a.tilesPerRow = (w + kM - 1) / kM;
    a.segments = n * h * a.tilesPerRow;
    a.mIsX = cin >= cout ? 1 : 0;
    const int mBlocks = a.mIsX ? (cin + kM - 1) / kM : 1;
    // M operand: 16 planes staged (rows beyond the channels read stale
    // planes and are dropped); N operand: its channels.
    a.nDim = a.mIsX ? cout : cin;
    a.xPlanes = a.mIsX ? std::min(16, cin / 8) : cin / 8;  // the last M block may hold fewer (set per block below)
    a.dPlanes = cout / 8;
    const uint32_t xStaged = a.mIsX ? 16u : (uint32_t)(cin / 8);
    const uint32_t dStaged = a.mIsX ? (uint32_t)(cout / 8) : 16u;
    a.xBytes = xStaged * kXPlane;
    a.stageBytes = a.xBytes + dStaged * kDPlane;
    a.accCols = (uint32_t)a.nDim;
    a.tmemCols = 32;
    while (a.tmemCols < 3u * a.accCols) a.tmemCols <<= 1;
    a.dw = dw;
    a.errorFlag = errorFlag;
    a.waitLimitNs = 1000000000ull;
    a.stages = 2;
    while (a.stages < kMaxStages && kHeader + (uint32_t)(a.stages + 1) * a.stageBytes <= 200u * 1024u) a.stages++;
    const uint32_t smemBytes = kHeader + (uint32_t)a.stages * a.stageBytes;
    if (smemBytes > 227u * 1024u) return cudaErrorNotSupported;
    a.mValid = a.mIsX ? std::min(kM, cin) : cout;
    int sms = 0, device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int perSm = std::max(1, std::min((int)(228u * 1024u / (smemBytes + 1024u)), (int)(512u / a.tmemCols)));
    const long long want = (long long)std::max(1, sms) * perSm * 2;
    const int splits = (int)std::max(1ll, std::min<long long>(a.segments, want / (3ll * mBlocks)));
    a.segPerBlock = (a.segments + splits - 1) / splits;
    const int grid = (a.segments + a.segPerBlock - 1) / a.segPerBlock;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(wgradTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    // M blocks of 128 input channels (224 = 128 + 96), one launch each.
    for (int mb = 0; mb < mBlocks; mb++) {
        WgradArgs b = a;
        if (a.mIsX) {
            const int channels = std::min(kM, cin - mb * kM);
            b.mBase = mb * kM;
            b.xPlanes = channels / 8;
            b.mValid = channels;
        }
        wgradTcKernel<<<dim3(grid, 3, 1), kThreads, smemBytes, stream>>>(xMap, dMap, b);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

}  // namespace rt
