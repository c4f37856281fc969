// tcgen05 implicit-GEMM 3x3 convolution (see rt_conv_tc.cuh).
//
// Persistent blocks (one per SM, or more when shared and tensor memory
// allow; 4 warps, or 8 + 1 for layers with fewer than 4 blocks per SM, see
// WarpLayout) walk over tiles of 128 output pixels. For every tile the
// input channels are taken in chunks of 16 or 32: all threads stage the
// chunk's halo (and, when the weights do not fit in shared memory for the
// whole kernel, the chunk's weights) with cp.async into one of two stages;
// one thread issues the chunk's 9 taps x (chunk / 16) MMAs of 128 x N x 16 and
// commits them to the stage's mbarrier, while the threads go on to stage
// the next chunk into the other stage. After a tile's last chunk the
// draining warps read the accumulators back from tensor memory (each warp 32
// lanes = 32 pixels and its share of the channel groups), add the bias,
// apply ReLU and store.
//
// Every wait on an mbarrier is bounded; past the bound the kernel stops its
// work, waits for its own copies, frees its tensor memory, sets *errorFlag
// and returns.
#include <algorithm>

#include <atomic>

#include "rt_conv_tc.cuh"

namespace rt {
namespace {

using bf16 = __nv_bfloat16;
constexpr int kTileM = 128;             // output pixels per tile (the MMA's M)
constexpr int kHaloW = kTileM + 2;      // halo pixels per row
// Warp layouts (template parameters of the kernel): DRAIN warps stage and
// drain; in the epilogue warp w < DRAIN reads tensor-memory lanes
// 32 * (w % 4) .. + 31 (the lanes a warp may access) and every DRAIN / 4-th
// group of 16 accumulator columns from 16 * (w / 4). With ISSUER = 1 an
// extra warp issues the MMAs and takes no part in the epilogue, so issuing a
// tile's MMAs overlaps the drain of the previous tile instead of delaying it
// (a block barrier waits for the slowest warp); with ISSUER = 0 thread 0
// issues. Layers that fit 4 or more blocks per SM use 4 warps (more blocks,
// less per-block overhead), the others 8 + 1.
template <int DRAIN, int ISSUER>
struct WarpLayout {
    static constexpr int kThreads = 32 * (DRAIN + ISSUER);
    static constexpr int kIssuer = ISSUER ? 32 * DRAIN : 0;
    static constexpr int kDrainWarps = DRAIN;
    static constexpr int kColumnStep = 16 * (DRAIN / 4);
};
constexpr uint32_t kHeaderBytes = 128;  // mbarriers and the tensor-memory address
constexpr uint32_t kMaxSmem = 227 * 1024;

static_assert(ummaInstrDescBf16(128, 64) == 0x08100490u, "instruction descriptor layout");

struct ConvTcArgs {
    const bf16* in;       // input, or the skip part (cin - lowChannels channels) of a concatenated input
    const bf16* low;      // upsampled part (nearest, from h/2 x w/2) of a concatenated input, or null
    int lowChannels;
    int n, h, w, cin;
    const bf16* weights;
    int reverseTaps;
    const float* bias;
    int cout;
    bf16* outB;
    float* outF;
    int relu, accumulate;
    int tiles, tilesPerRow;
    int kc;               // input channels per chunk (a multiple of 16 dividing cin)
    int resident;         // 1: all chunks' weights stay in shared memory
    int ring;             // 1: row strips over a 4-row ring of input rows (one chunk, resident weights)
    int stripRows;        // rows per strip in ring mode
    uint32_t weightBytes; // weight region: all chunks (resident) or two stages
    uint32_t haloBytes;   // one halo stage
    uint32_t tmemCols;
    uint32_t accCols;     // columns of one accumulator (two in ring mode)
    int* errorFlag;
};

__device__ __forceinline__ uint32_t smemAddress(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void mbarInit(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// mbarrier.try_wait suspends the thread until the phase completes or the
// hint (1 us) passes, so a completion wakes the waiters at once. A wait gives
// up one second (of %globaltimer, not a count of tries: a suspension may end
// early) after its first failed try.
__device__ __forceinline__ bool mbarTryWait(uint32_t bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase), "r"(1000u)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t globalTimerNs() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t kWaitLimitNs = 1000000000ull;
__device__ bool mbarWait(uint32_t bar, uint32_t phase) {
    if (mbarTryWait(bar, phase)) return true;
    const uint64_t deadline = globalTimerNs() + kWaitLimitNs;
    while (!mbarTryWait(bar, phase))
        if (globalTimerNs() > deadline) return false;
    return true;
}

__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void mmaBf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void mmaCommit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// The 9 taps x K MMAs of a tile (or of one channel chunk of it), K a
// compile-time constant: one thread issuing from a loop with a runtime trip
// count issued an MMA per ~155 SM cycles, fully unrolled per ~60 (the
// tensor pipe itself takes ~42 per 128 x N x 16 with N <= 64). aTap[t] is
// tap t's A offset and every step a 16-byte-unit offset from the bases.
template <int K>
__device__ __forceinline__ void issueTaps(uint32_t acc, uint64_t aBase, const uint32_t (&aTap)[9], uint32_t kStepA,
                                          uint64_t bBase, uint32_t tapStepB, uint32_t kStepB, uint32_t idesc,
                                          bool accumulateFirst) {
#pragma unroll
    for (int t = 0; t < 9; t++)
#pragma unroll
        for (int k = 0; k < K; k++)
            mmaBf16(acc, aBase + aTap[t] + (uint64_t)k * kStepA, bBase + (uint64_t)t * tapStepB + (uint64_t)k * kStepB,
                    idesc, (accumulateFirst || t > 0 || k > 0) ? 1u : 0u);
}
__device__ __forceinline__ void issueTapsK(int k, uint32_t acc, uint64_t aBase, const uint32_t (&aTap)[9],
                                           uint32_t kStepA, uint64_t bBase, uint32_t tapStepB, uint32_t kStepB,
                                           uint32_t idesc, bool accumulateFirst) {
#define RT_ISSUE_CASE(K) \
    case K: issueTaps<K>(acc, aBase, aTap, kStepA, bBase, tapStepB, kStepB, idesc, accumulateFirst); return;
    switch (k) {
        RT_ISSUE_CASE(1) RT_ISSUE_CASE(2) RT_ISSUE_CASE(3) RT_ISSUE_CASE(4) RT_ISSUE_CASE(5) RT_ISSUE_CASE(6)
        RT_ISSUE_CASE(7) RT_ISSUE_CASE(8) RT_ISSUE_CASE(9) RT_ISSUE_CASE(10) RT_ISSUE_CASE(11) RT_ISSUE_CASE(12)
        RT_ISSUE_CASE(13) RT_ISSUE_CASE(14)
        default: break;
    }
#undef RT_ISSUE_CASE
    // Wider chunks (cin above 224 held whole): the loop form.
    for (int t = 0; t < 9; t++)
        for (int j = 0; j < k; j++)
            mmaBf16(acc, aBase + aTap[t] + (uint64_t)j * kStepA, bBase + (uint64_t)t * tapStepB + (uint64_t)j * kStepB,
                    idesc, (accumulateFirst || t > 0 || j > 0) ? 1u : 0u);
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

template <int DRAIN, int ISSUER>
__global__ void __launch_bounds__(WarpLayout<DRAIN, ISSUER>::kThreads, DRAIN == 4 ? 4 : 2) convTcKernel(ConvTcArgs a) {
    using Layout = WarpLayout<DRAIN, ISSUER>;
    constexpr int kThreads = Layout::kThreads, kIssuer = Layout::kIssuer, kDrainWarps = Layout::kDrainWarps;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);          // two mbarriers
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(smem + 16);  // tensor-memory address
    unsigned char* wbuf = smem + kHeaderBytes;
    unsigned char* hbuf = wbuf + a.weightBytes;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int groups = a.kc / 8;          // 8-channel planes per chunk
    const int chunks = a.cin / a.kc;
    const uint32_t haloPlane = 3u * kHaloW * 16u;
    const uint32_t stageW = 9u * (uint32_t)a.kc * (uint32_t)a.cout * 2u;  // one chunk's weights
    const uint32_t bar0 = smemAddress(&bars[0]), bar1 = smemAddress(&bars[1]);

    if (tid == 0) {
        mbarInit(bar0, 1);
        mbarInit(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smemAddress(tmemSlot)),
                     "r"(a.tmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tcFenceBefore();
    __syncthreads();
    tcFenceAfter();
    const uint32_t tmem = *tmemSlot;
    const uint32_t idesc = ummaInstrDescBf16(kTileM, a.cout);

    // Stages one chunk's weights: [tap][plane][n], 16 bytes per entry.
    auto stageWeights = [&](int chunk, unsigned char* w) {
        const int vecs = 9 * groups * a.cout;
        for (int v = tid; v < vecs; v += kThreads) {
            const int nIdx = v % a.cout, g = (v / a.cout) % groups, t = v / (a.cout * groups);
            const int ts = a.reverseTaps ? 8 - t : t;
            const bf16* src = a.weights + ((size_t)ts * a.cout + nIdx) * a.cin + (size_t)chunk * a.kc + g * 8;
            cpAsync16(smemAddress(w + ((size_t)(t * groups + g) * a.cout + nIdx) * 16), src, true);
        }
    };
    // Stages one chunk of a tile's halo: [plane][row][pixel], zeros outside the image.
    auto stageHalo = [&](int tile, int chunk, unsigned char* halo) {
        const int xt = tile % a.tilesPerRow, rowIdx = tile / a.tilesPerRow;  // rowIdx = image * h + y
        const int y = rowIdx % a.h, x0 = xt * kTileM;
        const size_t imageBase = (size_t)(rowIdx - y) * a.w;  // first pixel of the image
        const int vecs = groups * 3 * kHaloW;
        for (int v = tid; v < vecs; v += kThreads) {
            const int p = v % kHaloW, r = (v / kHaloW) % 3, g = v / (3 * kHaloW);
            const int yy = y + r - 1, xx = x0 + p - 1;
            const bool ok = yy >= 0 && yy < a.h && xx >= 0 && xx < a.w;
            const int c = chunk * a.kc + g * 8;  // first channel of the 16-byte entry
            const bf16* src = a.in;
            if (ok) {
                if (c < a.lowChannels) {  // upsampled part: pixel (yy / 2, xx / 2) of the half-size input
                    const int img = (rowIdx - y) / a.h, hh = a.h >> 1, wh = a.w >> 1;
                    src = a.low + (((size_t)img * hh + (yy >> 1)) * wh + (xx >> 1)) * a.lowChannels + c;
                } else {
                    src = a.in + (imageBase + (size_t)yy * a.w + xx) * (a.cin - a.lowChannels) + (c - a.lowChannels);
                }
            }
            cpAsync16(smemAddress(halo + ((size_t)(g * 3 + r) * kHaloW + p) * 16), src, ok);
        }
    };

    // Ring mode: stages input row yy of image img (all channels) into ring
    // slot `slot`: [plane][slot][pixel], zeros outside the image.
    auto stageRow = [&](int img, int yy, int x0, int slot) {
        const int vecs = groups * kHaloW;
        const bool rowOk = yy >= 0 && yy < a.h;
        for (int v = tid; v < vecs; v += kThreads) {
            const int p = v % kHaloW, g = v / kHaloW;
            const int xx = x0 + p - 1;
            const bool ok = rowOk && xx >= 0 && xx < a.w;
            const int c = g * 8;
            const bf16* src = a.in;
            if (ok) {
                if (c < a.lowChannels) {
                    const int hh = a.h >> 1, wh = a.w >> 1;
                    src = a.low + (((size_t)img * hh + (yy >> 1)) * wh + (xx >> 1)) * a.lowChannels + c;
                } else {
                    src = a.in + (((size_t)img * a.h + yy) * a.w + xx) * (a.cin - a.lowChannels) + (c - a.lowChannels);
                }
            }
            cpAsync16(smemAddress(hbuf + ((size_t)(g * 4 + slot) * kHaloW + p) * 16), src, ok);
        }
    };
    // Epilogue of one tile (row rowIdx = image * h + y, first column x0):
    // accumulators from tensor memory, bias, ReLU, store.
    auto epilogue = [&](int rowIdx, int x0, uint32_t column) {
        tcFenceAfter();
        if (warp >= kDrainWarps) {  // the issuing warp: only the barrier below
            tcFenceBefore();
            __syncthreads();
            return;
        }
        const int quarter = warp & 3, half = warp >> 2;
        const int x = x0 + quarter * 32 + lane;
        const bool inside = x < a.w;
        const size_t pix = (size_t)rowIdx * a.w + (size_t)x;
        for (int cb = 16 * half; cb < a.cout; cb += Layout::kColumnStep) {
            uint32_t r[16];
            tmemLoad16(tmem + ((uint32_t)(quarter * 32) << 16) + column + (uint32_t)cb, r);
            if (!inside) continue;
            float v[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                float sum = __uint_as_float(r[j]) + (a.bias ? a.bias[cb + j] : 0.0f);
                v[j] = a.relu ? fmaxf(sum, 0.0f) : sum;
            }
            if (a.outF) {
                float4* o = reinterpret_cast<float4*>(a.outF + pix * a.cout + cb);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float4 add = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                    if (a.accumulate) {
                        float4 old = o[q];
                        add = make_float4(old.x + add.x, old.y + add.y, old.z + add.z, old.w + add.w);
                    }
                    o[q] = add;
                }
            } else {
                uint4 packed[2];
                uint32_t* words = reinterpret_cast<uint32_t*>(packed);
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    __nv_bfloat162 pair = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    words[j] = *reinterpret_cast<uint32_t*>(&pair);
                }
                uint4* o = reinterpret_cast<uint4*>(a.outB + pix * a.cout + cb);
                o[0] = packed[0];
                o[1] = packed[1];
            }
        }
        tcFenceBefore();
        __syncthreads();
    };

    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    bool failed = false;

    if (a.ring) {
        // Row strips: a unit is (image, column tile, block of stripRows rows);
        // each tile stages only the row two below it while its MMAs run.
        const int strips = (a.h + a.stripRows - 1) / a.stripRows;
        const int units = a.n * a.tilesPerRow * strips;
        const uint32_t ringPlane = 4u * kHaloW * 16u;
        bool weightsStaged = false;
        for (int u = blockIdx.x; u < units && !failed; u += gridDim.x) {
            const int strip = u % strips, xt = (u / strips) % a.tilesPerRow, img = u / (strips * a.tilesPerRow);
            const int y0 = strip * a.stripRows, y1 = min(a.h, y0 + a.stripRows), x0 = xt * kTileM;
            if (!weightsStaged) { stageWeights(0, wbuf); weightsStaged = true; }
            for (int r = y0 - 1; r <= y0 + 1; r++) stageRow(img, r, x0, r & 3);
            cpAsyncCommit();
            // Tile y accumulates into tensor-memory half y & 1; the epilogue
            // of tile y - 1 runs while tile y's MMAs execute.
            for (int y = y0; y <= y1 && !failed; y++) {
                if (y > y0) {
                    // Tile y - 1's MMAs read rows y - 2 .. y; wait for them
                    // before slot (y + 2) & 3 (row y - 2) is overwritten.
                    const int b = (y - 1) & 1;
                    const bool ok = mbarWait(b ? bar1 : bar0, phase[b]);
                    phase[b] ^= 1u;
                    if (__syncthreads_or(!ok)) { failed = true; break; }
                }
                if (y < y1) {
                    if (y + 1 < y1) stageRow(img, y + 2, x0, (y + 2) & 3);
                    cpAsyncCommit();
                    cpAsyncWait<1>();
                    fenceProxyAsync();
                    __syncthreads();
                    if (tid == kIssuer) {
                        tcFenceAfter();
                        // Descriptors as base + offset in 16-byte units: the
                        // start address is the low 14-bit field and every
                        // operand lies in shared memory (< 256 KB), so the
                        // sum never carries into the other fields.
                        const uint64_t aBase = ummaSmemDesc(smemAddress(hbuf), ringPlane, 128u);
                        const uint64_t bBase = ummaSmemDesc(smemAddress(wbuf), (uint32_t)a.cout * 16u, 128u);
                        const uint32_t acc = tmem + (uint32_t)(y & 1) * a.accCols;
                        uint32_t aTap[9];
                        for (int t = 0; t < 9; t++)
                            aTap[t] = (uint32_t)(((y + t / 3 - 1) & 3) * kHaloW + t % 3);
                        issueTapsK(a.kc / 16, acc, aBase, aTap, 2u * 4u * kHaloW, bBase, (uint32_t)(groups * a.cout),
                                   2u * (uint32_t)a.cout, idesc, false);
                        mmaCommit((y & 1) ? bar1 : bar0);
                    }
                }
                if (y > y0) epilogue(img * a.h + y - 1, x0, (uint32_t)((y - 1) & 1) * a.accCols);
            }
        }
    }
    auto waitStage = [&](int s) -> bool {
        bool ok = true;
        if (pending[s]) {
            ok = mbarWait(s ? bar1 : bar0, phase[s]);
            phase[s] ^= 1u;
            pending[s] = false;
        }
        return ok;
    };

    int step = 0;
    int tile = a.ring ? a.tiles : blockIdx.x;
    if (tile < a.tiles) {
        if (a.resident)
            for (int c = 0; c < chunks; c++) stageWeights(c, wbuf + (size_t)c * stageW);
        else
            stageWeights(0, wbuf);
        stageHalo(tile, 0, hbuf);
        cpAsyncCommit();
    }
    for (; tile < a.tiles && !failed; tile += gridDim.x) {
        for (int c = 0; c < chunks; c++, step++) {
            const int stage = step & 1, other = stage ^ 1;
            int nextTile = tile, nextChunk = c + 1;
            if (nextChunk == chunks) { nextTile = tile + gridDim.x; nextChunk = 0; }
            const bool more = nextTile < a.tiles;
            if (more) {
                // The other stage is free once the MMAs that read it are done.
                const bool ok = waitStage(other);
                if (__syncthreads_or(!ok)) { failed = true; break; }
                if (!a.resident) stageWeights(nextChunk, wbuf + (size_t)other * stageW);
                stageHalo(nextTile, nextChunk, hbuf + (size_t)other * a.haloBytes);
                cpAsyncCommit();
                cpAsyncWait<1>();
            } else {
                cpAsyncWait<0>();
            }
            fenceProxyAsync();
            __syncthreads();
            if (tid == kIssuer) {
                tcFenceAfter();
                // Descriptors as base + offset in 16-byte units (see the
                // ring loop above).
                const uint64_t aBase = ummaSmemDesc(smemAddress(hbuf + (size_t)stage * a.haloBytes), haloPlane, 128u);
                const uint64_t bBase = ummaSmemDesc(
                    smemAddress(a.resident ? wbuf + (size_t)c * stageW : wbuf + (size_t)stage * stageW),
                    (uint32_t)a.cout * 16u, 128u);
                uint32_t aTap[9];
                for (int t = 0; t < 9; t++) aTap[t] = (uint32_t)((t / 3) * kHaloW + t % 3);
                issueTapsK(a.kc / 16, tmem, aBase, aTap, 2u * 3u * kHaloW, bBase, (uint32_t)(groups * a.cout),
                           2u * (uint32_t)a.cout, idesc, c > 0);
                mmaCommit(stage ? bar1 : bar0);
            }
            pending[stage] = true;
        }
        if (failed) break;
        // Accumulators of this tile: wait for the last chunk's MMAs (the
        // other stage's, if still outstanding, completed before them).
        {
            const int last = (step - 1) & 1;
            bool ok = waitStage(last ^ 1);
            ok = waitStage(last) && ok;
            if (__syncthreads_or(!ok)) { failed = true; break; }
        }
        epilogue(tile / a.tilesPerRow, (tile % a.tilesPerRow) * kTileM, 0u);
    }
    cpAsyncWait<0>();
    tcFenceBefore();
    __syncthreads();
    if (failed && tid == 0) atomicExch(a.errorFlag, 1);
    if (warp == 0) {
        tcFenceAfter();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(a.tmemCols)
                     : "memory");
    }
}

int deviceSms() {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms > 0 ? sms : 1;
}

}  // namespace

static std::atomic<int> g_convPath{0};
static std::atomic<long long> g_pipeLaunches{0}, g_singleLaunches{0};
void setConvPath(int mode) { g_convPath.store(mode); }
int convPath() { return g_convPath.load(); }
static std::atomic<bool> g_convPipeReference{false};
void setConvPipeReference(bool on) { g_convPipeReference.store(on); }
bool convPipeReference() { return g_convPipeReference.load(); }
void convLaunchCounts(long long* pipe, long long* single) {
    if (pipe) *pipe = g_pipeLaunches.load();
    if (single) *single = g_singleLaunches.load();
}

namespace {
// Low-resolution tap (a, b) of output parity (py, px) collects the full taps
// (dy, dx) with floor((py + dy - 1) / 2) = a - 1 and floor((px + dx - 1) / 2)
// = b - 1: nearest upsampling maps upsampled pixel 2i + t to low pixel i.
__global__ void combineUpsampledWeightsKernel(const bf16* w, int cout, int cin, int lowChannels, bf16* lowW,
                                              bf16* skipW) {
    const int skipC = cin - lowChannels;
    const long long nLow = 9ll * 4 * cout * lowChannels, nSkip = 9ll * cout * skipC;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nLow + nSkip;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < nLow) {
            const int ci = (int)(i % lowChannels);
            const int row = (int)((i / lowChannels) % (4 * cout));
            const int tap = (int)(i / lowChannels / (4 * cout));
            const int blk = row / cout, c = row % cout, py = blk >> 1, px = blk & 1;
            const int a = tap / 3, b = tap % 3;
            float sum = 0.0f;
            for (int dy = 0; dy < 3; dy++) {
                if (((py + dy + 1) >> 1) != a) continue;  // floor((py + dy - 1) / 2) + 1
                for (int dx = 0; dx < 3; dx++) {
                    if (((px + dx + 1) >> 1) != b) continue;
                    sum += __bfloat162float(w[((size_t)(dy * 3 + dx) * cout + c) * cin + ci]);
                }
            }
            lowW[i] = __float2bfloat16(sum);
        } else {
            const long long j = i - nLow;
            const int ci = (int)(j % skipC);
            const int c = (int)((j / skipC) % cout);
            const int tap = (int)(j / skipC / cout);
            skipW[j] = w[((size_t)tap * cout + c) * cin + lowChannels + ci];
        }
    }
}
}  // namespace

cudaError_t combineUpsampledWeights(const bf16* weights, int cout, int cin, int lowChannels, bf16* lowWeights,
                                    bf16* skipWeights, cudaStream_t stream) {
    if (!weights || !lowWeights || !skipWeights || lowChannels <= 0 || lowChannels >= cin) return cudaErrorInvalidValue;
    combineUpsampledWeightsKernel<<<296, 256, 0, stream>>>(weights, cout, cin, lowChannels, lowWeights, skipWeights);
    return cudaGetLastError();
}

bool upsampledSplitSupported(int cin, int cout, int lowChannels) {
    return lowChannels > 0 && lowChannels < cin && cout <= 64 && convPipePreferred(lowChannels, 4 * cout, 0) &&
           convPipePreferred(cin - lowChannels, cout, 0);
}

cudaError_t convTc(const bf16* in, const bf16* low, int lowChannels, int n, int h, int w, int cin,
                   const bf16* weights, bool reverseTaps, const float* bias, int cout, bf16* outB, float* outF,
                   bool relu, bool accumulate, int* errorFlag, cudaStream_t stream, const bf16* upAddend,
                   const ConvHead* head, bool planarOut) {
    if (upAddend || head || planarOut) {  // the two-pass decoder form, a fused head: pipelined kernel only
        if (low || !convPipePreferred(cin, cout, 0)) return cudaErrorNotSupported;
        cudaError_t e = convPipe(in, nullptr, 0, n, h, w, cin, weights, reverseTaps, bias, cout, outB, outF, relu,
                                 accumulate, errorFlag, stream, nullptr, upAddend, head, planarOut);
        if (e == cudaSuccess) g_pipeLaunches++;
        return e;
    }
    // The warp-specialised TMA form where its shared memory allows (see
    // rt_conv_pipe.cu); this kernel for the layers with the largest weights.
    if (g_convPath.load() == 0 && convPipePreferred(cin, cout, low ? lowChannels : 0)) {
        cudaError_t e = convPipe(in, low, lowChannels, n, h, w, cin, weights, reverseTaps, bias, cout, outB, outF,
                                 relu, accumulate, errorFlag, stream);
        if (e != cudaErrorNotSupported) {
            g_pipeLaunches++;
            return e;
        }
    }
    g_singleLaunches++;
    if (n < 1 || h < 1 || w < 1 || cin < 16 || cin % 16 || cout < 16 || cout % 16 || cout > 256 ||
        (!outB && !outF) || !errorFlag || (low && (lowChannels < 16 || lowChannels % 16 || lowChannels >= cin ||
                                                   h % 2 || w % 2)))
        return cudaErrorInvalidValue;
    static bool configured = false;
    if (!configured) {
        void (*kernels[2])(ConvTcArgs) = {convTcKernel<4, 0>, convTcKernel<8, 1>};
        for (auto k : kernels) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            if (e != cudaSuccess) return e;
        }
        configured = true;
    }
    ConvTcArgs a{};
    a.in = in; a.low = low; a.lowChannels = low ? lowChannels : 0;
    a.n = n; a.h = h; a.w = w; a.cin = cin;
    a.weights = weights; a.reverseTaps = reverseTaps ? 1 : 0;
    a.bias = bias; a.cout = cout; a.outB = outB; a.outF = outF;
    a.relu = relu ? 1 : 0; a.accumulate = accumulate ? 1 : 0;
    a.tilesPerRow = (w + kTileM - 1) / kTileM;
    a.tiles = n * h * a.tilesPerRow;
    a.errorFlag = errorFlag;
    // Weights stay in shared memory when they fit beside two halo stages;
    // the chunk is the largest multiple of 16 dividing cin that still fits
    // (one chunk per tile where possible: fewer rounds of staging). Otherwise
    // weights and halo are staged per 16-channel chunk.
    const uint32_t fullWeights = 9u * (uint32_t)cin * (uint32_t)cout * 2u;
    const uint32_t haloPerChannel = 3u * kHaloW * 2u;
    const uint32_t ringBytes = 4u * kHaloW * 2u * (uint32_t)cin;
    a.resident = 0;
    a.ring = kHeaderBytes + fullWeights + ringBytes <= 220u * 1024u;
    for (int kc = a.ring ? 16 : cin; kc >= 16; kc -= 16) {
        if (cin % kc) continue;
        if (kHeaderBytes + fullWeights + 2u * haloPerChannel * (uint32_t)kc <= 220u * 1024u) {
            a.kc = kc;
            a.resident = 1;
            break;
        }
    }
    if (a.ring) {
        a.kc = cin;
        a.resident = 1;
        a.weightBytes = fullWeights;
        a.haloBytes = ringBytes / 2u;  // the ring takes the two halo stages' room
    } else if (a.resident) {
        a.weightBytes = fullWeights;
        a.haloBytes = haloPerChannel * (uint32_t)a.kc;
    } else {
        a.kc = 16;
        a.weightBytes = 2u * 9u * 16u * (uint32_t)cout * 2u;
        a.haloBytes = haloPerChannel * (uint32_t)a.kc;
    }
    const uint32_t smemBytes = kHeaderBytes + a.weightBytes + 2u * a.haloBytes;
    if (smemBytes > kMaxSmem) return cudaErrorInvalidValue;
    a.accCols = 32;
    while (a.accCols < (uint32_t)cout) a.accCols <<= 1;
    a.tmemCols = a.ring ? 2u * a.accCols : a.accCols;  // ring mode: two accumulators
    // Blocks per SM: shared memory (228 KB per SM, 1 KB reserved per block)
    // and the 512 columns of tensor memory.
    // Layers that fit 4 or more blocks of 4 warps per SM keep 4 warps; the
    // others run 8 draining warps and an issuing warp (measured per layer:
    // 16->32 at full resolution 102 against 122 us, 80->32 578 against 480).
    int perSm = (int)((228u * 1024u) / (smemBytes + 1024u));
    perSm = std::max(1, std::min({perSm, (int)(512u / a.tmemCols), 8}));
    const bool wide = perSm < 4;
    if (wide) perSm = std::min(perSm, 2048 / WarpLayout<8, 1>::kThreads);
    int units = a.tiles;
    if (a.ring) {
        a.stripRows = balancedStripRows((long long)n * a.tilesPerRow, h, (long long)deviceSms() * perSm);
        units = n * a.tilesPerRow * ((h + a.stripRows - 1) / a.stripRows);
    }
    const int grid = std::min(units, deviceSms() * perSm);
    if (wide)
        convTcKernel<8, 1><<<grid, WarpLayout<8, 1>::kThreads, smemBytes, stream>>>(a);
    else
        convTcKernel<4, 0><<<grid, WarpLayout<4, 0>::kThreads, smemBytes, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace rt
