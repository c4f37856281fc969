// 3x3 convolutions of the learned denoiser on the fifth-generation tensor
// cores (tcgen05.mma, BF16 operands in shared memory, FP32 accumulators in
// tensor memory).
//
// Implicit GEMM: D[pixel][n] = sum over taps and input channels of
// A[pixel][k] * B[n][k], with A the input shifted by the tap. A block owns
// 128 consecutive output pixels of one image row (the MMA's M = 128) and all
// N output channels. The input halo of the tile (3 rows x 130 pixels x a
// chunk of input channels) sits in shared memory as planes of 8 channels, 16
// bytes per pixel, which is the no-swizzle K-major operand layout: core
// matrices of 8 pixels x 8 channels, 8-pixel groups 128 bytes apart (SBO),
// the two 8-channel halves of an MMA's K = 16 one plane apart (LBO). Each of
// the 9 taps is the same buffer read from a start address shifted by the
// tap's pixel offset, so no im2col copy is made. Weights are K-major
// [tap][n][k] in the same plane form.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace rt {

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5 = 1), BF16 A and B (bits 7-9 and 10-12 = 1), both K-major (bits 15 and
// 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t ummaInstrDescBf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Shared-memory matrix descriptor, no swizzle: start address, leading-
// dimension byte offset (LBO) and stride-dimension byte offset (SBO), each in
// 16-byte units in 14-bit fields at bits 0, 16 and 32; descriptor version 1
// (bit 46); base offset, LBO mode and layout type (bits 49-63) zero.
__host__ __device__ constexpr uint64_t ummaSmemDesc(uint32_t address, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((address >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// out[p][n] = act(bias[n] + sum_tap,k in[p + off(tap)][k] * w[tap'][n][k]) over
// NHWC BF16 input with Cin channels; w is [9][Cout][Cin] BF16 (K-major) and
// tap' = 8 - tap when reverseTaps (the data gradient reads the forward
// weights [tap][cin][cout] this way). Cin and Cout multiples of 16, Cout <=
// 256. Writes BF16 (outB) or FP32 (outF, added to when accumulate). errorFlag
// is set if a wait on the tensor cores runs past its limit.
// With `low` set, the input is the concatenation [upsample2(low), in] read
// in place: channels [0, lowChannels) from low (h/2 x w/2, nearest) and the
// rest from `in` (cin - lowChannels channels per pixel); h and w even.
// A 1x1 output head fused into a convolution's epilogue (pipelined form
// only): for the output pixels inside crop (w x h, row stride w), out[pixel]
// [k] = max(expm1(b[k] + sum_c bf16(act[c]) * wt[c * 3 + k]), 0) for k < 3,
// summed over the channels in order as a separate 1x1 pass over the BF16
// activations would; the convolution's own activations are not stored.
struct ConvHead {
    const float* wt;  // [cout][3]
    const float* b;   // [3]
    float* out;       // [h][w][3]
    int h, w;
};

// upAddend (optional, pipelined form only): the upsampled half of a decoder
// convolution computed at half resolution (see combineUpsampledWeights),
// 4 blocks of cout channels per low pixel, added before bias and ReLU; it is
// stored as planes of 8 channels over the low pixels, element (low pixel q,
// channel c of the 4 cout) at ((c / 8) * lowPixels + q) * 8 + c % 8, which
// is what a convolution with planarOut (pipelined form only) writes: a warp's
// 32 pixels then store 512 contiguous bytes per plane instead of 16 bytes per
// pixel at the pixel stride.
cudaError_t convTc(const __nv_bfloat16* in, const __nv_bfloat16* low, int lowChannels, int n, int h, int w, int cin,
                   const __nv_bfloat16* weights, bool reverseTaps, const float* bias, int cout, __nv_bfloat16* outB,
                   float* outF, bool relu, bool accumulate, int* errorFlag, cudaStream_t stream,
                   const __nv_bfloat16* upAddend = nullptr, const ConvHead* head = nullptr, bool planarOut = false);

// A decoder convolution over [upsample2(low), skip] as two convolutions:
// the low half at low resolution with 4 blocks of cout output channels, one
// per output-pixel parity (py, px) (nearest upsampling makes each output
// pixel's 3x3 window over the upsampled image a 3x3 window over the low
// image with some taps merged), and the skip half at full resolution, whose
// epilogue adds the first's block (see convTc's upAddend). This writes the
// low half's weights [tap'][4 * cout][lowChannels] (tap' over the low
// image's 3x3 window, block (py, px) = sum of the full taps that land
// there) and the skip half's [tap][cout][cin - lowChannels], both BF16 (the
// sums in FP32), from the forward weights [tap][cout][cin].
cudaError_t combineUpsampledWeights(const __nv_bfloat16* weights, int cout, int cin, int lowChannels,
                                    __nv_bfloat16* lowWeights, __nv_bfloat16* skipWeights, cudaStream_t stream);
// Whether the two-pass form runs on the pipelined kernel for this layer.
bool upsampledSplitSupported(int cin, int cout, int lowChannels);

// Rows per strip for kernels whose blocks walk (image, column tile, strip)
// units: the length (1-64 rows) that minimises the rows the busiest of
// `blocks` blocks stages, ceil(units / blocks) strips of s + 2 rows each (a
// strip stages one halo row above and below); the longest of equals.
inline int balancedStripRows(long long columns, int h, long long blocks) {
    int best = 1;
    long long bestCost = -1;
    for (int s = 1; s <= 64; s++) {
        const long long units = columns * ((h + s - 1) / s);
        const long long cost = (units + blocks - 1) / blocks * (s + 2);
        if (bestCost < 0 || cost <= bestCost) { bestCost = cost; best = s; }
        if (s >= h) break;
    }
    return best;
}

// Which kernel convTc runs: 0 (default) the pipelined form wherever it
// applies, 1 always the kernel above (process-wide; for comparisons).
void setConvPath(int mode);
int convPath();
// The pipelined kernel's reference form (default off): every layer's MMAs
// issued tap by tap per output tile over input rows staged as planes of 8
// channels, instead of the stacked-row issue and swizzled slabs; results are
// identical, for comparison.
void setConvPipeReference(bool on);
bool convPipeReference();
// Convolutions run so far by the pipelined and by the single-role kernel.
void convLaunchCounts(long long* pipe, long long* single);

// Test hooks of the pipelined form (convPipe): zero values keep the defaults.
struct ConvPipeTest {
    unsigned long long waitLimitNs;  // bound of every wait (default one second)
    int probe;                       // 1: the MMA issuer first waits on a barrier nothing completes
    int ring;                        // ring rows (3..16)
    int stripRows;                   // rows per strip
    int nAcc;                        // tensor-memory accumulators (2..8)
    unsigned long long* stats;       // device array of 6 wait/lifetime sums in ns (see rt_conv_pipe.cu)
    int blocksPerSm;                 // fewer blocks per SM than shared memory allows (each then gets a longer ring)
    int issuers;                     // MMA issuers per block: 0 chosen per layer, 1, or 2 (sharing the ring)
    int stacked;                     // 0 chosen per layer, 1 tap-per-tile issue, 2 stacked-row issue
    int planes;                      // 1: input rows staged as planes of 8 channels (no swizzled slabs)
    int epilogueWarps;               // 4: no second set of epilogue warps (0 chosen per layer)
};

// The same convolution as convTc, warp-specialised and fed by TMA (input
// rows in a ring of shared-memory slots, weights resident): for Cout in {16,
// 32, 48, 64, 80, 96, 128} when the weights and a ring of 3 rows fit in shared
// memory. Returns cudaErrorNotSupported (before any launch) for other
// shapes. Same arguments as convTc, plus optional test hooks.
bool convPipeSupported(int cin, int cout, int lowChannels);
// Whether convTc hands the layer to convPipe (path 0): when a ring of at
// least 4 rows fits beside the weights. With only the three rows a tile
// reads, the producer cannot run ahead of the MMAs and the single-role
// kernel is faster (1080p decoder layers 112->48 and 160->64: 287 and 368 us
// pipelined against 207 and 210 us).
bool convPipePreferred(int cin, int cout, int lowChannels);
uint32_t convPipeSmemBytes(int cin, int cout, int lowChannels, int ring);
cudaError_t convPipe(const __nv_bfloat16* in, const __nv_bfloat16* low, int lowChannels, int n, int h, int w, int cin,
                     const __nv_bfloat16* weights, bool reverseTaps, const float* bias, int cout,
                     __nv_bfloat16* outB, float* outF, bool relu, bool accumulate, int* errorFlag,
                     cudaStream_t stream, const ConvPipeTest* test = nullptr,
                     const __nv_bfloat16* upAddend = nullptr, const ConvHead* head = nullptr, bool planarOut = false);

// Weight gradient on tcgen05 (rt_wgrad_tc.cu): dw[tap][ci][co] += sum_p
// x[p + off(tap)][ci] dy[p][co] over NHWC BF16 x (cin channels) and dy (cout
// channels), dw FP32 [9][cin][cout]. cin, cout multiples of 16, cout <= 128,
// cin <= 256. Returns cudaErrorNotSupported (before any launch) otherwise.
bool wgradTcSupported(int cin, int cout);
cudaError_t wgradTc(const __nv_bfloat16* x, const __nv_bfloat16* dy, int n, int h, int w, int cin, int cout, float* dw,
                    int* errorFlag, cudaStream_t stream);

// Runs the pipelined kernel once with a wait that must run out (2 ms limit
// on a barrier nothing completes), then once normally: 1 when the first
// launch reported the timeout through its error flag without a CUDA error
// and the second produced the right output, else 0.
int convPipeWaitProbe();

}  // namespace rt
