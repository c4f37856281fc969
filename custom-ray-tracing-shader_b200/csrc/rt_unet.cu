// Learned denoiser (see rt_unet.cuh): kernels, forward, backward, Adam.
//
// Activations are NHWC BF16 with channel counts that are multiples of 16.
//   forward      out[p][co] = b[co] + sum_tap,ci x[p + off(tap)][ci] w[tap][ci][co]
//                on the fifth-generation tensor cores (convTc, rt_conv_tc.cu)
//                with K-major weights wT[tap][co][ci]
//   data grad    convTc on dY with B[ci][co] = w[8 - tap][ci][co]: the forward
//                weights read with the taps reversed
//   weight grad  dw[tap][ci][co] = sum_p x[p + off(tap)][ci] dY[p][co] on
//                the tensor cores (wgradTc, rt_wgrad_tc.cu; the 16x16x16
//                warp-level MMA kernel wgradKernel when the single-role
//                convolution path is selected)
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

#include "rt_common.cuh"
#include "rt_conv_tc.cuh"
#include "rt_unet.cuh"

namespace rt {
namespace {

using bf16 = __nv_bfloat16;
using namespace nvcuda;

constexpr int kTileX = 16, kTileY = 4;
constexpr int kWidths[5] = {32, 48, 64, 96, 128};
constexpr int kInputChannels = 10, kInputPadded = 16, kOutChannels = 3;

inline int blocksFor(long long n, int b) { return (int)((n + b - 1) / b); }

// ---- weight gradient ----
// Block: one tap, 16 input channels, CT output channels, a chunk of 16-pixel
// row segments; per-warp shared staging; partial sums added to dw atomically.
template <int CT>
__global__ void __launch_bounds__(128) wgradKernel(const bf16* __restrict__ x, const bf16* __restrict__ dy, int N,
                                                   int H, int W, int Cin, int Cout, int segmentsPerBlock,
                                                   float* dw) {
    __shared__ __align__(32) bf16 sX[4][16][16];
    __shared__ __align__(32) bf16 sD[4][16][CT];
    __shared__ __align__(32) float sAcc[4][16][CT];
    const int tap = blockIdx.y % 9, ci0 = (blockIdx.y / 9) * 16, co0 = blockIdx.z * CT;
    const int ky = tap / 3 - 1, kx = tap % 3 - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int segsPerRow = (W + 15) / 16;
    const long long segments = (long long)N * H * segsPerRow;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[CT / 16];
#pragma unroll
    for (int f = 0; f < CT / 16; f++) wmma::fill_fragment(acc[f], 0.0f);
    const long long begin = (long long)blockIdx.x * segmentsPerBlock;
    for (long long s = begin + warp; s < begin + segmentsPerBlock && s < segments; s += 4) {
        int xs = (int)(s % segsPerRow) * 16;
        long long row = s / segsPerRow;
        int y = (int)(row % H), n = (int)(row / H);
        // x[n][y + ky][xs + px + kx][ci0 .. ci0 + 15], zero outside the image.
        for (int k = lane; k < 32; k += 32) {
            int px = k >> 1, half = k & 1;
            int yy = y + ky, xx = xs + px + kx;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < H && xx >= 0 && xx < W && xs + px < W)
                v = *reinterpret_cast<const uint4*>(x + (((size_t)n * H + yy) * W + xx) * Cin + ci0 + half * 8);
            *reinterpret_cast<uint4*>(&sX[warp][px][half * 8]) = v;
        }
        constexpr int perPix = CT / 8;
        for (int k = lane; k < 16 * perPix; k += 32) {
            int px = k / perPix, part = k % perPix;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (xs + px < W)
                v = *reinterpret_cast<const uint4*>(dy + (((size_t)n * H + y) * W + xs + px) * Cout + co0 + part * 8);
            *reinterpret_cast<uint4*>(&sD[warp][px][part * 8]) = v;
        }
        __syncwarp();
        wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> a;  // (ci, pixel) = sX[pixel][ci]
        wmma::load_matrix_sync(a, &sX[warp][0][0], 16);
#pragma unroll
        for (int f = 0; f < CT / 16; f++) {
            wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> b;
            wmma::load_matrix_sync(b, &sD[warp][0][f * 16], CT);
            wmma::mma_sync(acc[f], a, b, acc[f]);
        }
        __syncwarp();
    }
#pragma unroll
    for (int f = 0; f < CT / 16; f++) wmma::store_matrix_sync(&sAcc[warp][0][f * 16], acc[f], CT, wmma::mem_row_major);
    __syncthreads();
    for (int k = threadIdx.x; k < 16 * CT; k += blockDim.x) {
        int ci = k / CT, c = k % CT;
        float v = sAcc[0][ci][c] + sAcc[1][ci][c] + sAcc[2][ci][c] + sAcc[3][ci][c];
        if (v != 0.0f) atomicAdd(&dw[((size_t)tap * Cin + ci0 + ci) * Cout + co0 + c], v);
    }
}

// ---- elementwise and reshaping kernels ----
__global__ void inputKernel(const float* aov, int n, int h, int w, int H, int W, bf16* x0, const int* batch,
                            const unsigned char* flips) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)n * H * W;
    if (i >= total) return;
    int X = (int)(i % W), Y = (int)((i / W) % H), b = (int)(i / ((long long)W * H));
    float v[kInputPadded] = {};
    {
        // The padded frame beyond w x h repeats the edge pixels.
        int src = batch ? batch[b] : b;
        int sx = min(X, w - 1), sy = min(Y, h - 1);
        if (flips) { if (flips[b] & 1) sx = w - 1 - sx; if (flips[b] & 2) sy = h - 1 - sy; }
        const float* a = aov + (((size_t)src * h + sy) * w + sx) * kInputChannels;
        v[0] = log1pf(fmaxf(a[0], 0.0f)); v[1] = log1pf(fmaxf(a[1], 0.0f)); v[2] = log1pf(fmaxf(a[2], 0.0f));
        v[3] = a[3]; v[4] = a[4]; v[5] = a[5];
        v[6] = a[6]; v[7] = a[7]; v[8] = a[8];
        v[9] = log1pf(fmaxf(a[9], 0.0f));
    }
    uint4 packed[2];
    uint32_t* words = reinterpret_cast<uint32_t*>(packed);
#pragma unroll
    for (int j = 0; j < kInputPadded / 2; j++) {
        __nv_bfloat162 pair = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        words[j] = *reinterpret_cast<uint32_t*>(&pair);
    }
    uint4* o = reinterpret_cast<uint4*>(x0 + (size_t)i * kInputPadded);
    o[0] = packed[0];
    o[1] = packed[1];
}
__global__ void targetKernel(const float* target, int n, int h, int w, float* out, const int* batch,
                             const unsigned char* flips) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)n * h * w;
    if (i >= total) return;
    int X = (int)(i % w), Y = (int)((i / w) % h), b = (int)(i / ((long long)w * h));
    int src = batch ? batch[b] : b;
    int sx = X, sy = Y;
    if (flips) { if (flips[b] & 1) sx = w - 1 - X; if (flips[b] & 2) sy = h - 1 - Y; }
    const float* t = target + (((size_t)src * h + sy) * w + sx) * 3;
    for (int c = 0; c < 3; c++) out[(size_t)i * 3 + c] = log1pf(fmaxf(t[c], 0.0f));
}
// 2x2 average pooling, 8 channels per thread (16-byte loads and stores).
__global__ void poolKernel(const bf16* in, int N, int H, int W, int C, bf16* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int Ho = H / 2, Wo = W / 2, C8 = C / 8;
    long long total = (long long)N * Ho * Wo * C8;
    if (i >= total) return;
    int c = (int)(i % C8) * 8;
    long long p = i / C8;
    int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), n = (int)(p / ((long long)Wo * Ho));
    const bf16* b = in + (((size_t)n * H + 2 * y) * W + 2 * x) * C + c;
    uint4 q[4] = {*reinterpret_cast<const uint4*>(b), *reinterpret_cast<const uint4*>(b + C),
                  *reinterpret_cast<const uint4*>(b + (size_t)W * C), *reinterpret_cast<const uint4*>(b + (size_t)W * C + C)};
    const bf16* e[4] = {reinterpret_cast<const bf16*>(&q[0]), reinterpret_cast<const bf16*>(&q[1]),
                        reinterpret_cast<const bf16*>(&q[2]), reinterpret_cast<const bf16*>(&q[3])};
    uint4 r;
    bf16* o = reinterpret_cast<bf16*>(&r);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        float s = __bfloat162float(e[0][j]) + __bfloat162float(e[1][j]) + __bfloat162float(e[2][j]) +
                  __bfloat162float(e[3][j]);
        o[j] = __float2bfloat16(0.25f * s);
    }
    *reinterpret_cast<uint4*>(out + (size_t)p * C + c) = r;
}
__global__ void poolBackwardKernel(const float* dOut, int N, int H, int W, int C, float* dIn, int accumulate) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)N * H * W * C;
    if (i >= total) return;
    int c = (int)(i % C);
    long long p = i / C;
    int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((long long)W * H));
    float v = 0.25f * dOut[(((size_t)n * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
    dIn[i] = accumulate ? dIn[i] + v : v;
}
// out = concat(upsample2(low), skip) along channels.
__global__ void upConcatKernel(const bf16* low, int Cl, const bf16* skip, int Cs, int N, int H, int W, bf16* out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int C = Cl + Cs;
    long long total = (long long)N * H * W * C;
    if (i >= total) return;
    int c = (int)(i % C);
    long long p = i / C;
    int x = (int)(p % W), y = (int)((p / W) % H), n = (int)(p / ((long long)W * H));
    out[i] = c < Cl ? low[(((size_t)n * (H / 2) + y / 2) * (W / 2) + x / 2) * Cl + c]
                    : skip[(((size_t)n * H + y) * W + x) * Cs + (c - Cl)];
}
// Backward of upConcat: gradient of low (summed over 2x2) and of skip.
__global__ void upConcatBackwardLowKernel(const float* dOut, int Cl, int Cs, int N, int H, int W, float* dLow) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int Hl = H / 2, Wl = W / 2, C = Cl + Cs;
    long long total = (long long)N * Hl * Wl * Cl;
    if (i >= total) return;
    int c = (int)(i % Cl);
    long long p = i / Cl;
    int x = (int)(p % Wl), y = (int)((p / Wl) % Hl), n = (int)(p / ((long long)Wl * Hl));
    const float* d = dOut + (((size_t)n * H + 2 * y) * W + 2 * x) * C + c;
    dLow[i] = d[0] + d[C] + d[(size_t)W * C] + d[(size_t)W * C + C];
}
__global__ void upConcatBackwardSkipKernel(const float* dOut, int Cl, int Cs, long long pixels, float* dSkip) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels * Cs) return;
    int c = (int)(i % Cs);
    long long p = i / Cs;
    dSkip[i] = dOut[p * (Cl + Cs) + Cl + c];
}
__global__ void reluMaskKernel(const float* dY, const bf16* y, long long count, bf16* dPre) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    dPre[i] = __float2bfloat16(__bfloat162float(y[i]) > 0.0f ? dY[i] : 0.0f);
}
__global__ void biasGradKernel(const bf16* dPre, long long pixels, int C, float* db) {
    int c = threadIdx.x % C;
    int lanesPerBlock = blockDim.x / C;
    int slot = threadIdx.x / C;
    if (slot >= lanesPerBlock) return;
    float s = 0.0f;
    for (long long p = (long long)blockIdx.x * lanesPerBlock + slot; p < pixels; p += (long long)gridDim.x * lanesPerBlock)
        s += __bfloat162float(dPre[p * C + c]);
    atomicAdd(&db[c], s);
}
// K-major copy for the forward convolution: wT[tap][co][ci] = w[tap][ci][co].
__global__ void transposeKernel(const bf16* w, int Cin, int Cout, bf16* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * Cin * Cout) return;
    int ci = i % Cin, co = (i / Cin) % Cout, tap = i / (Cin * Cout);
    out[i] = w[((size_t)tap * Cin + ci) * Cout + co];
}
__global__ void toBf16Kernel(const float* in, size_t count, bf16* out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = __float2bfloat16(in[i]);
}
// 1x1 output layer, forward: pred[p][k] = b[k] + sum_c d[p][c] w[c][k].
__global__ void outForwardKernel(const bf16* d, long long pixels, int C, const float* w, const float* b, float* pred) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    float s[kOutChannels] = {b[0], b[1], b[2]};
    for (int c8 = 0; c8 < C; c8 += 8) {
        uint4 q = *reinterpret_cast<const uint4*>(d + p * C + c8);
        const bf16* e = reinterpret_cast<const bf16*>(&q);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            float v = __bfloat162float(e[j]);
            for (int k = 0; k < kOutChannels; k++) s[k] += v * w[(c8 + j) * kOutChannels + k];
        }
    }
    for (int k = 0; k < kOutChannels; k++) pred[p * kOutChannels + k] = s[k];
}
// L1 loss in log space: loss += |pred - t| / count; dPred = sign / count.
__global__ void lossKernel(const float* pred, const float* t, long long count, float* dPred, float* loss) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < count) {
        float d = pred[i] - t[i];
        l = fabsf(d);
        dPred[i] = (d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f)) / (float)count;
    }
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l / (float)count);
}
// 1x1 output layer, backward.
__global__ void outBackwardKernel(const bf16* d, const float* dPred, long long pixels, int C, const float* w,
                                  float* dW, float* dB, float* dD) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float g[kOutChannels] = {0, 0, 0};
    if (p < pixels)
        for (int k = 0; k < kOutChannels; k++) g[k] = dPred[p * kOutChannels + k];
    for (int k = 0; k < kOutChannels; k++) {
        float v = g[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
        if ((threadIdx.x & 31) == 0 && v != 0.0f) atomicAdd(&dB[k], v);
    }
    for (int c = 0; c < C; c++) {
        float x = p < pixels ? __bfloat162float(d[p * C + c]) : 0.0f;
        float dd = 0.0f;
        for (int k = 0; k < kOutChannels; k++) {
            float v = x * g[k];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, off);
            if ((threadIdx.x & 31) == 0 && v != 0.0f) atomicAdd(&dW[c * kOutChannels + k], v);
            dd += g[k] * w[c * kOutChannels + k];
        }
        if (p < pixels) dD[p * C + c] = dd;
    }
}
__global__ void adamKernel(float* p, const float* g, float* m, float* v, size_t count, float lr, float b1, float b2,
                           float eps, float c1, float c2) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}
// Network output (log space, padded frame) to linear radiance (w x h x 3).
// Network input straight from the running sums: the AOVs of RtxReadAovs
// (sum / samples, normalised normal, distance / samples), then the input
// transform of inputKernel, for every pixel of the padded frame (beyond w x h
// the edge pixels repeat).
__global__ void sumsInputKernel(const float* sums, const float* depthSums, unsigned samples, int h, int w, int H,
                                int W, bf16* x0) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)H * W) return;
    const int X = (int)(i % W), Y = (int)(i / W);
    const size_t src = (size_t)min(Y, h - 1) * w + min(X, w - 1);
    const float* a = sums + src * 10;
    const float inv = 1.0f / (float)samples;
    const float3 c = scale(v3(a[0], a[1], a[2]), inv), al = scale(v3(a[3], a[4], a[5]), inv);
    const float3 nr = normalize(v3(a[6], a[7], a[8]));
    const float depth = depthSums[src] * inv;
    float v[kInputPadded] = {};
    v[0] = log1pf(fmaxf(c.x, 0.0f)); v[1] = log1pf(fmaxf(c.y, 0.0f)); v[2] = log1pf(fmaxf(c.z, 0.0f));
    v[3] = al.x; v[4] = al.y; v[5] = al.z;
    v[6] = nr.x; v[7] = nr.y; v[8] = nr.z;
    v[9] = log1pf(fmaxf(depth, 0.0f));
    uint4 packed[2];
    uint32_t* words = reinterpret_cast<uint32_t*>(packed);
#pragma unroll
    for (int j = 0; j < kInputPadded / 2; j++) {
        __nv_bfloat162 pair = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        words[j] = *reinterpret_cast<uint32_t*>(&pair);
    }
    uint4* o = reinterpret_cast<uint4*>(x0 + (size_t)i * kInputPadded);
    o[0] = packed[0];
    o[1] = packed[1];
}
// Output layer and crop in one pass: the 1x1 convolution of outForwardKernel
// (same summation order) for the pixels inside w x h, then expm1 and the
// clamp of outputKernel.
__global__ void outputFusedKernel(const bf16* d, int H, int W, int h, int w, int C, const float* wt, const float* b,
                                  float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int x = i % w, y = i / w;
    const long long p = (long long)y * W + x;
    float s[kOutChannels] = {b[0], b[1], b[2]};
    for (int c8 = 0; c8 < C; c8 += 8) {
        uint4 q = *reinterpret_cast<const uint4*>(d + p * C + c8);
        const bf16* e = reinterpret_cast<const bf16*>(&q);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            float v = __bfloat162float(e[j]);
            for (int k = 0; k < kOutChannels; k++) s[k] += v * wt[(c8 + j) * kOutChannels + k];
        }
    }
    for (int k = 0; k < kOutChannels; k++) out[(size_t)i * 3 + k] = fmaxf(expm1f(s[k]), 0.0f);
}

__global__ void outputKernel(const float* pred, int H, int W, int h, int w, float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    int x = i % w, y = i / w;
    const float* p = pred + ((size_t)y * W + x) * kOutChannels;
    for (int k = 0; k < kOutChannels; k++) out[(size_t)i * 3 + k] = fmaxf(expm1f(p[k]), 0.0f);
}

template <int CT>
cudaError_t launchWgrad(const bf16* x, const bf16* dy, int N, int H, int W, int Cin, int Cout, float* dw, cudaStream_t s) {
    long long segments = (long long)N * H * ((W + 15) / 16);
    int chunks = (int)std::min<long long>(64, std::max<long long>(1, segments / 64));
    int per = (int)((segments + chunks - 1) / chunks);
    dim3 grid(chunks, 9 * (Cin / 16), Cout / CT);
    wgradKernel<CT><<<grid, 128, 0, s>>>(x, dy, N, H, W, Cin, Cout, per, dw);
    return cudaGetLastError();
}
// Weight gradient: the tcgen05 kernel (rt_wgrad_tc.cu) unless the
// single-role convolution path is selected (RtxSetConvPath(1)), then the
// warp-level MMA kernel above.
cudaError_t wgrad(const bf16* x, const bf16* dy, int N, int H, int W, int Cin, int Cout, float* dw, int* errorFlag,
                  cudaStream_t s) {
    if (convPath() == 0 && wgradTcSupported(Cin, Cout)) {
        cudaError_t e = wgradTc(x, dy, N, H, W, Cin, Cout, dw, errorFlag, s);
        if (e != cudaErrorNotSupported) return e;
    }
    if (Cout % 64 == 0) return launchWgrad<64>(x, dy, N, H, W, Cin, Cout, dw, s);
    if (Cout % 48 == 0) return launchWgrad<48>(x, dy, N, H, W, Cin, Cout, dw, s);
    if (Cout % 32 == 0) return launchWgrad<32>(x, dy, N, H, W, Cin, Cout, dw, s);
    return launchWgrad<16>(x, dy, N, H, W, Cin, Cout, dw, s);
}

}  // namespace

// Activations and gradients for one (n, H, W) configuration.
struct Unet::Activations {
    int n = 0, H = 0, W = 0;
    bool training = false;
    bf16* x0 = nullptr;
    bf16* a[18] = {};        // outputs of the 18 3x3 layers
    bf16* pool[4] = {};      // pooled encoder outputs (levels 1..4 inputs)
    bf16* cat[4] = {};       // decoder inputs: concat(upsample(lower), skip) at levels 3..0
    // Two-pass form of the decoders' first convolutions (inference): the
    // upsampled half at half resolution (4 parity blocks of cout channels)
    // and each layer's combined weights (low half, skip half).
    bf16* upHalf = nullptr;
    bf16* upWeights[4] = {};
    bf16* skipWeights[4] = {};
    float* pred = nullptr;   // network output, log space
    float* target = nullptr; // log-space target
    float* dPred = nullptr;
    float* dAct[18] = {};    // fp32 gradients of layer outputs
    float* dCat[4] = {};
    float* dPool[4] = {};
    bf16* dPre = nullptr;    // scratch: gradient at the pre-activation, bf16
    float* loss = nullptr;
    int* batch = nullptr;
    unsigned char* flips = nullptr;
    std::vector<void*> owned;
    template <class T>
    cudaError_t make(T*& p, size_t count) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(count, 1));
        if (e == cudaSuccess) owned.push_back(p);
        return e;
    }
    ~Activations() {
        for (void* p : owned) cudaFree(p);
    }
};

namespace {
// Layer table: 10 encoder/bottleneck layers then 8 decoder layers.
void layerTable(std::vector<UnetLayer>& layers, size_t& params) {
    int cin[18], cout[18];
    int prev = kInputPadded, k = 0;
    for (int l = 0; l < 5; l++) {
        cin[k] = prev; cout[k] = kWidths[l]; k++;
        cin[k] = kWidths[l]; cout[k] = kWidths[l]; k++;
        prev = kWidths[l];
    }
    for (int l = 3; l >= 0; l--) {
        cin[k] = prev + kWidths[l]; cout[k] = kWidths[l]; k++;
        cin[k] = kWidths[l]; cout[k] = kWidths[l]; k++;
        prev = kWidths[l];
    }
    params = 0;
    for (int i = 0; i < 18; i++) {
        UnetLayer L{cin[i], cout[i], params, params + (size_t)9 * cin[i] * cout[i]};
        params = L.bOffset + cout[i];
        layers.push_back(L);
    }
    UnetLayer out{kWidths[0], kOutChannels, params, params + (size_t)kWidths[0] * kOutChannels};
    params = out.bOffset + kOutChannels;
    layers.push_back(out);
}
}  // namespace

Unet::Unet(unsigned seed) {
    layerTable(layers_, params_);
    std::vector<float> host(params_, 0.0f);
    std::mt19937 rng(seed);
    for (size_t l = 0; l < layers_.size(); l++) {
        const UnetLayer& L = layers_[l];
        bool out = l + 1 == layers_.size();
        int fanIn = (out ? 1 : 9) * (l == 0 ? kInputChannels : L.cin);
        std::normal_distribution<float> dist(0.0f, std::sqrt((out ? 1.0f : 2.0f) / (float)fanIn));
        size_t nw = L.bOffset - L.wOffset;
        for (size_t i = 0; i < nw; i++) {
            float v = dist(rng);
            if (l == 0) {  // padding input channels carry zeros: their weights stay zero
                size_t ci = (i / L.cout) % L.cin;
                if ((int)ci >= kInputChannels) v = 0.0f;
            }
            host[L.wOffset + i] = v;
        }
    }
    cudaMalloc(&master_, sizeof(float) * params_);
    cudaMalloc(&grad_, sizeof(float) * params_);
    cudaMalloc(&adamM_, sizeof(float) * params_);
    cudaMalloc(&adamV_, sizeof(float) * params_);
    cudaMalloc(&wbf_, sizeof(bf16) * params_);
    cudaMalloc(&wT_, sizeof(bf16) * params_);
    cudaMalloc(&convError_, sizeof(int));
    // Every copy and fill goes through stream_: it is non-blocking, so it is
    // not ordered after work on the legacy default stream.
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    cudaMemsetAsync(convError_, 0, sizeof(int), stream_);
    cudaMemcpyAsync(master_, host.data(), sizeof(float) * params_, cudaMemcpyHostToDevice, stream_);
    cudaMemsetAsync(adamM_, 0, sizeof(float) * params_, stream_);
    cudaMemsetAsync(adamV_, 0, sizeof(float) * params_, stream_);
    syncWeights(stream_);
    cudaStreamSynchronize(stream_);
}

Unet::~Unet() {
    delete act_;
    cudaFree(master_); cudaFree(grad_); cudaFree(adamM_); cudaFree(adamV_); cudaFree(wbf_); cudaFree(wT_); cudaFree(convError_);
    if (stream_) cudaStreamDestroy(stream_);
}

cudaError_t Unet::syncWeights(cudaStream_t s) {
    toBf16Kernel<<<blocksFor((long long)params_, 256), 256, 0, s>>>(master_, params_, wbf_);
    for (size_t l = 0; l + 1 < layers_.size(); l++) {
        const UnetLayer& L = layers_[l];
        transposeKernel<<<blocksFor(9LL * L.cin * L.cout, 256), 256, 0, s>>>(wbf_ + L.wOffset, L.cin, L.cout, wT_ + L.wOffset);
    }
    return cudaGetLastError();
}

cudaError_t Unet::checkConvolutions(std::string& error) {
    int flag = 0;
    cudaError_t e = cudaMemcpy(&flag, convError_, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return e;
    if (!flag) return cudaSuccess;
    e = cudaMemsetAsync(convError_, 0, sizeof(int), stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return e;
    error = "tensor-core convolution stopped: a wait on the tensor cores ran past its limit";
    return cudaErrorLaunchTimeout;
}

cudaError_t Unet::getParams(float* host) const {
    cudaError_t e = cudaMemcpyAsync(host, master_, sizeof(float) * params_, cudaMemcpyDeviceToHost, stream_);
    return e == cudaSuccess ? cudaStreamSynchronize(stream_) : e;
}
cudaError_t Unet::setParams(const float* host) {
    cudaError_t e = cudaMemcpyAsync(master_, host, sizeof(float) * params_, cudaMemcpyHostToDevice, stream_);
    if (e != cudaSuccess) return e;
    e = syncWeights(stream_);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(stream_);
}

cudaError_t Unet::ensure(int n, int h, int w, bool training) {
    int H = (h + 15) / 16 * 16, W = (w + 15) / 16 * 16;
    if (act_ && act_->n == n && act_->H == H && act_->W == W && (act_->training || !training)) return cudaSuccess;
    delete act_;
    act_ = new Activations();
    Activations& A = *act_;
    A.n = n; A.H = H; A.W = W; A.training = training;
    cudaError_t e = cudaSuccess;
    auto px = [&](int level) { return (size_t)n * (H >> level) * (W >> level); };
    if ((e = A.make(A.x0, px(0) * kInputPadded)) != cudaSuccess) return e;
    for (int k = 0; k < 18; k++) {
        int level = k < 10 ? k / 2 : 3 - (k - 10) / 2;
        if ((e = A.make(A.a[k], px(level) * layers_[k].cout)) != cudaSuccess) return e;
        if (training && (e = A.make(A.dAct[k], px(level) * layers_[k].cout)) != cudaSuccess) return e;
    }
    for (int l = 1; l <= 4; l++) {
        if ((e = A.make(A.pool[l - 1], px(l) * kWidths[l - 1])) != cudaSuccess) return e;
        if (training && (e = A.make(A.dPool[l - 1], px(l) * kWidths[l - 1])) != cudaSuccess) return e;
    }
    size_t upHalf = 0;
    for (int j = 0; j < 4; j++) {  // decoder level 3 - j
        int level = 3 - j;
        const UnetLayer& L = layers_[10 + 2 * j];
        const int Cl = layers_[9 + 2 * j].cout;
        if (upsampledSplitSupported(L.cin, L.cout, Cl)) {
            upHalf = std::max(upHalf, px(level) * L.cout);  // (H / 2) x (W / 2) x 4 cout
            if ((e = A.make(A.upWeights[j], (size_t)9 * 4 * L.cout * Cl)) != cudaSuccess) return e;
            if ((e = A.make(A.skipWeights[j], (size_t)9 * L.cout * (L.cin - Cl))) != cudaSuccess) return e;
        }
        if (training && (e = A.make(A.cat[j], px(level) * layers_[10 + 2 * j].cin)) != cudaSuccess) return e;
        if (training && (e = A.make(A.dCat[j], px(level) * layers_[10 + 2 * j].cin)) != cudaSuccess) return e;
    }
    if (upHalf && (e = A.make(A.upHalf, upHalf)) != cudaSuccess) return e;
    if ((e = A.make(A.pred, px(0) * kOutChannels)) != cudaSuccess) return e;
    if (training) {
        if ((e = A.make(A.target, px(0) * kOutChannels)) != cudaSuccess) return e;
        if ((e = A.make(A.dPred, px(0) * kOutChannels)) != cudaSuccess) return e;
        if ((e = A.make(A.dPre, px(0) * 128)) != cudaSuccess) return e;
        if ((e = A.make(A.loss, 1)) != cudaSuccess) return e;
        if ((e = A.make(A.batch, n)) != cudaSuccess) return e;
        if ((e = A.make(A.flips, n)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t Unet::forward(cudaStream_t s, bool training, bool outputLayer, const ConvHead* head, bool* headDone) {
    if (headDone) *headDone = false;
    Activations& A = *act_;
    const int n = A.n;
    cudaError_t e;
    const bf16* x = A.x0;
    int k = 0;
    for (int l = 0; l < 5; l++) {
        int H = A.H >> l, W = A.W >> l;
        if (l > 0) {
            int C = kWidths[l - 1];
            poolKernel<<<blocksFor((long long)n * H * W * (C / 8), 256), 256, 0, s>>>(A.a[k - 1], n, H * 2, W * 2, C, A.pool[l - 1]);
            x = A.pool[l - 1];
        }
        for (int r = 0; r < 2; r++, k++) {
            const UnetLayer& L = layers_[k];
            if ((e = convTc(x, nullptr, 0, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset, L.cout, A.a[k], nullptr, true, false, convError_, s)) != cudaSuccess) return e;
            x = A.a[k];
        }
    }
    for (int j = 0; j < 4; j++) {
        int level = 3 - j, H = A.H >> level, W = A.W >> level;
        int Cl = layers_[k - 1].cout, Cs = kWidths[level];
        const bf16* low = A.a[k - 1];
        const bf16* skip = A.a[2 * level + 1];
        for (int r = 0; r < 2; r++, k++) {
            const UnetLayer& L = layers_[k];
            if (r == 0 && training) {
                // The weight gradient reads the concatenated input: keep it.
                upConcatKernel<<<blocksFor((long long)n * H * W * (Cl + Cs), 256), 256, 0, s>>>(low, Cl, skip, Cs, n, H, W, A.cat[j]);
                e = convTc(A.cat[j], nullptr, 0, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset, L.cout, A.a[k], nullptr, true, false, convError_, s);
            } else if (r == 0 && A.upWeights[j] && convPath() == 0) {
                // Inference, two passes: the upsampled half at half
                // resolution (4 parity blocks), then the skip half adding it.
                e = combineUpsampledWeights(wT_ + L.wOffset, L.cout, L.cin, Cl, A.upWeights[j], A.skipWeights[j], s);
                if (e == cudaSuccess)
                    e = convTc(low, nullptr, 0, n, H / 2, W / 2, Cl, A.upWeights[j], false, nullptr, 4 * L.cout, A.upHalf,
                               nullptr, false, false, convError_, s, nullptr, nullptr, true);
                if (e == cudaSuccess)
                    e = convTc(skip, nullptr, 0, n, H, W, Cs, A.skipWeights[j], false, master_ + L.bOffset, L.cout, A.a[k],
                               nullptr, true, false, convError_, s, A.upHalf);
            } else if (r == 0) {
                // Inference: the convolution reads [upsample(low), skip] in place.
                e = convTc(skip, low, Cl, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset, L.cout, A.a[k], nullptr, true, false, convError_, s);
            } else if (k == 17 && head && !training && convPath() == 0 && convPipePreferred(L.cin, L.cout, 0)) {
                // The last convolution with the output head in its epilogue.
                e = convTc(A.a[k - 1], nullptr, 0, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset, L.cout,
                           nullptr, nullptr, true, false, convError_, s, nullptr, head);
                if (e == cudaSuccess && headDone) *headDone = true;
                if (e == cudaErrorNotSupported)
                    e = convTc(A.a[k - 1], nullptr, 0, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset,
                               L.cout, A.a[k], nullptr, true, false, convError_, s);
            } else {
                e = convTc(A.a[k - 1], nullptr, 0, n, H, W, L.cin, wT_ + L.wOffset, false, master_ + L.bOffset, L.cout, A.a[k], nullptr, true, false, convError_, s);
            }
            if (e != cudaSuccess) return e;
        }
    }
    if (!outputLayer) return cudaGetLastError();
    const UnetLayer& O = layers_[18];
    long long pixels = (long long)n * A.H * A.W;
    outForwardKernel<<<blocksFor(pixels, 128), 128, 0, s>>>(A.a[17], pixels, O.cin, master_ + O.wOffset, master_ + O.bOffset, A.pred);
    return cudaGetLastError();
}

cudaError_t Unet::backward(cudaStream_t s) {
    Activations& A = *act_;
    const int n = A.n;
    cudaError_t e;
    cudaMemsetAsync(grad_, 0, sizeof(float) * params_, s);
    const UnetLayer& O = layers_[18];
    long long pixels0 = (long long)n * A.H * A.W;
    outBackwardKernel<<<blocksFor(pixels0, 128), 128, 0, s>>>(A.a[17], A.dPred, pixels0, O.cin, master_ + O.wOffset,
                                                             grad_ + O.wOffset, grad_ + O.bOffset, A.dAct[17]);
    // Backward through one 3x3 layer k whose output gradient is dAct[k];
    // writes the input gradient to dIn (fp32) unless dIn is null.
    auto layerBack = [&](int k, const bf16* input, int H, int W, float* dIn, bool accumulate) -> cudaError_t {
        const UnetLayer& L = layers_[k];
        long long count = (long long)n * H * W * L.cout;
        reluMaskKernel<<<blocksFor(count, 256), 256, 0, s>>>(A.dAct[k], A.a[k], count, A.dPre);
        int per = std::max(1, 256 / L.cout);
        biasGradKernel<<<std::min<long long>(1024, blocksFor((long long)n * H * W, per)), per * L.cout, 0, s>>>(
            A.dPre, (long long)n * H * W, L.cout, grad_ + L.bOffset);
        cudaError_t err = wgrad(input, A.dPre, n, H, W, L.cin, L.cout, grad_ + L.wOffset, convError_, s);
        if (err != cudaSuccess) return err;
        if (dIn) return convTc(A.dPre, nullptr, 0, n, H, W, L.cout, wbf_ + L.wOffset, true, nullptr, L.cin, nullptr, dIn, false, accumulate, convError_, s);
        return cudaSuccess;
    };
    int k = 17;
    for (int j = 3; j >= 0; j--) {  // decoder level 3 - j, from the top (level 0) down
        int level = 3 - j, H = A.H >> level, W = A.W >> level;
        if ((e = layerBack(k, A.a[k - 1], H, W, A.dAct[k - 1], false)) != cudaSuccess) return e;
        k--;
        if ((e = layerBack(k, A.cat[j], H, W, A.dCat[j], false)) != cudaSuccess) return e;
        k--;
        int Cl = layers_[k].cout, Cs = kWidths[level];  // layers_[k]: the layer below (its output was upsampled)
        upConcatBackwardLowKernel<<<blocksFor((long long)n * (H / 2) * (W / 2) * Cl, 256), 256, 0, s>>>(
            A.dCat[j], Cl, Cs, n, H, W, A.dAct[k]);
        // skip gradient into the encoder output of this level (dAct[2*level+1]) — set here, pooled part added below
        upConcatBackwardSkipKernel<<<blocksFor((long long)n * H * W * Cs, 256), 256, 0, s>>>(
            A.dCat[j], Cl, Cs, (long long)n * H * W, A.dAct[2 * level + 1]);
    }
    // Bottleneck and encoder: k = 9 down to 0.
    for (int l = 4; l >= 0; l--) {
        int H = A.H >> l, W = A.W >> l;
        const bf16* in1 = l == 0 ? A.x0 : A.pool[l - 1];
        // second conv of level l: input a[2l], output a[2l+1]
        if ((e = layerBack(2 * l + 1, A.a[2 * l], H, W, A.dAct[2 * l], false)) != cudaSuccess) return e;
        // first conv of level l: input in1
        if ((e = layerBack(2 * l, in1, H, W, l == 0 ? nullptr : A.dPool[l - 1], false)) != cudaSuccess) return e;
        if (l > 0) {
            int C = kWidths[l - 1];
            // encoder output of level l-1 receives the pooled gradient plus its skip gradient
            poolBackwardKernel<<<blocksFor((long long)n * H * 2 * W * 2 * C, 256), 256, 0, s>>>(
                A.dPool[l - 1], n, H * 2, W * 2, C, A.dAct[2 * (l - 1) + 1], 1);
        }
    }
    return cudaGetLastError();
}

cudaError_t Unet::lossAndGradient(const float* aovs, const float* targets, int n, int h, int w, float* loss, float* grads,
                                  std::string& error) {
    if (h % 16 || w % 16) { error = "training crops must be multiples of 16 pixels"; return cudaErrorInvalidValue; }
    cudaError_t e = ensure(n, h, w, true);
    if (e != cudaSuccess) return e;
    Activations& A = *act_;
    float *dA = nullptr, *dT = nullptr;
    size_t px = (size_t)n * h * w;
    if ((e = cudaMalloc(&dA, sizeof(float) * px * kInputChannels)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&dT, sizeof(float) * px * 3)) != cudaSuccess) { cudaFree(dA); return e; }
    cudaMemcpyAsync(dA, aovs, sizeof(float) * px * kInputChannels, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(dT, targets, sizeof(float) * px * 3, cudaMemcpyHostToDevice, stream_);
    inputKernel<<<blocksFor((long long)px, 256), 256, 0, stream_>>>(dA, n, h, w, A.H, A.W, A.x0, nullptr, nullptr);
    targetKernel<<<blocksFor((long long)px, 256), 256, 0, stream_>>>(dT, n, h, w, A.target, nullptr, nullptr);
    cudaMemsetAsync(A.loss, 0, sizeof(float), stream_);
    if ((e = forward(stream_, true)) == cudaSuccess) {
        lossKernel<<<blocksFor((long long)px * 3, 256), 256, 0, stream_>>>(A.pred, A.target, (long long)px * 3, A.dPred, A.loss);
        e = backward(stream_);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss, A.loss, sizeof(float), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess && grads) e = cudaMemcpyAsync(grads, grad_, sizeof(float) * params_, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e == cudaSuccess) e = checkConvolutions(error);
    cudaFree(dA); cudaFree(dT);
    return e;
}

cudaError_t Unet::train(const float* aovs, const float* targets, int count, int h, int w, int steps, int batch,
                        float lr, unsigned seed, float* losses, std::string& error) {
    if (h % 16 || w % 16) { error = "training crops must be multiples of 16 pixels"; return cudaErrorInvalidValue; }
    if (batch < 1 || count < 1) { error = "empty training set"; return cudaErrorInvalidValue; }
    cudaError_t e = ensure(batch, h, w, true);
    if (e != cudaSuccess) return e;
    Activations& A = *act_;
    float *dA = nullptr, *dT = nullptr;
    size_t px = (size_t)count * h * w;
    if ((e = cudaMalloc(&dA, sizeof(float) * px * kInputChannels)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&dT, sizeof(float) * px * 3)) != cudaSuccess) { cudaFree(dA); return e; }
    cudaMemcpyAsync(dA, aovs, sizeof(float) * px * kInputChannels, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(dT, targets, sizeof(float) * px * 3, cudaMemcpyHostToDevice, stream_);
    std::mt19937 rng(seed);
    std::vector<int> idx(batch);
    std::vector<unsigned char> flips(batch);
    std::vector<float> lossHost(steps, 0.0f);
    float* dLosses = nullptr;
    if ((e = cudaMalloc(&dLosses, sizeof(float) * std::max(steps, 1))) != cudaSuccess) { cudaFree(dA); cudaFree(dT); return e; }
    cudaMemsetAsync(dLosses, 0, sizeof(float) * std::max(steps, 1), stream_);
    const size_t bpx = (size_t)batch * h * w;
    for (int step = 0; step < steps && e == cudaSuccess; step++) {
        for (int b = 0; b < batch; b++) { idx[b] = (int)(rng() % (unsigned)count); flips[b] = (unsigned char)(rng() & 3u); }
        cudaMemcpyAsync(A.batch, idx.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(A.flips, flips.data(), batch, cudaMemcpyHostToDevice, stream_);
        inputKernel<<<blocksFor((long long)bpx, 256), 256, 0, stream_>>>(dA, batch, h, w, A.H, A.W, A.x0, A.batch, A.flips);
        targetKernel<<<blocksFor((long long)bpx, 256), 256, 0, stream_>>>(dT, batch, h, w, A.target, A.batch, A.flips);
        if ((e = forward(stream_, true)) != cudaSuccess) break;
        lossKernel<<<blocksFor((long long)bpx * 3, 256), 256, 0, stream_>>>(A.pred, A.target, (long long)bpx * 3, A.dPred, dLosses + step);
        if ((e = backward(stream_)) != cudaSuccess) break;
        adamStep_++;
        const float b1 = 0.9f, b2 = 0.999f;
        float c1 = 1.0f - std::pow(b1, (float)adamStep_), c2 = 1.0f - std::pow(b2, (float)adamStep_);
        adamKernel<<<blocksFor((long long)params_, 256), 256, 0, stream_>>>(master_, grad_, adamM_, adamV_, params_, lr, b1, b2, 1e-8f, c1, c2);
        if ((e = syncWeights(stream_)) != cudaSuccess) break;
        // The tiny host copies above wait for the stream; keep them ordered.
        if ((step & 63) == 63) e = cudaStreamSynchronize(stream_);
    }
    if (e == cudaSuccess && losses) e = cudaMemcpyAsync(losses, dLosses, sizeof(float) * steps, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e == cudaSuccess) e = checkConvolutions(error);
    cudaFree(dA); cudaFree(dT); cudaFree(dLosses);
    return e;
}

cudaError_t Unet::inferFromSums(const float* sums, const float* depthSums, unsigned samples, int h, int w,
                                float* radiance, cudaStream_t s) {
    cudaError_t e = ensure(1, h, w, false);
    if (e != cudaSuccess) return e;
    Activations& A = *act_;
    sumsInputKernel<<<blocksFor((long long)A.H * A.W, 256), 256, 0, s>>>(sums, depthSums, samples, h, w, A.H, A.W, A.x0);
    const UnetLayer& O = layers_[18];
    const ConvHead head{master_ + O.wOffset, master_ + O.bOffset, radiance, h, w};
    bool fused = false;
    if ((e = forward(s, false, false, &head, &fused)) != cudaSuccess) return e;
    if (!fused)
        outputFusedKernel<<<blocksFor((long long)w * h, 256), 256, 0, s>>>(A.a[17], A.H, A.W, h, w, O.cin,
                                                                          master_ + O.wOffset, master_ + O.bOffset,
                                                                          radiance);
    return cudaGetLastError();
}

cudaError_t Unet::inferDevice(const float* aovs, int h, int w, float* radiance, cudaStream_t s, std::string&) {
    cudaError_t e = ensure(1, h, w, false);
    if (e != cudaSuccess) return e;
    Activations& A = *act_;
    inputKernel<<<blocksFor((long long)A.H * A.W, 256), 256, 0, s>>>(aovs, 1, h, w, A.H, A.W, A.x0, nullptr, nullptr);
    if ((e = forward(s, false)) != cudaSuccess) return e;
    outputKernel<<<blocksFor((long long)w * h, 256), 256, 0, s>>>(A.pred, A.H, A.W, h, w, radiance);
    return cudaGetLastError();
}

// Checkpoint: "RTUNET01", parameter count (u64), Adam step (i64), optimiser
// state flag (u64), FP32 parameters, then Adam m and v when the flag is set.
cudaError_t Unet::save(const char* path, bool optimizerState, std::string& error) const {
    std::vector<float> host(params_ * (optimizerState ? 3 : 1));
    cudaError_t e = cudaMemcpyAsync(host.data(), master_, sizeof(float) * params_, cudaMemcpyDeviceToHost, stream_);
    if (optimizerState) {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host.data() + params_, adamM_, sizeof(float) * params_, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host.data() + 2 * params_, adamV_, sizeof(float) * params_, cudaMemcpyDeviceToHost, stream_);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return e;
    FILE* f = std::fopen(path, "wb");
    if (!f) { error = std::string("cannot write ") + path; return cudaErrorInvalidValue; }
    const char magic[8] = {'R', 'T', 'U', 'N', 'E', 'T', '0', '1'};
    unsigned long long count = params_, state = optimizerState ? 1 : 0;
    long long step = optimizerState ? adamStep_ : 0;
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&count, 8, 1, f) == 1 && std::fwrite(&step, 8, 1, f) == 1 &&
              std::fwrite(&state, 8, 1, f) == 1 && std::fwrite(host.data(), sizeof(float), host.size(), f) == host.size();
    ok = std::fclose(f) == 0 && ok;
    if (!ok) { error = std::string("short write to ") + path; return cudaErrorInvalidValue; }
    return cudaSuccess;
}

cudaError_t Unet::load(const char* path, std::string& error) {
    FILE* f = std::fopen(path, "rb");
    if (!f) { error = std::string("cannot read ") + path; return cudaErrorInvalidValue; }
    char magic[8];
    unsigned long long count = 0, state = 0;
    long long step = 0;
    std::vector<float> host;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "RTUNET01", 8) == 0 && std::fread(&count, 8, 1, f) == 1 &&
              count == params_ && std::fread(&step, 8, 1, f) == 1 && std::fread(&state, 8, 1, f) == 1 && state <= 1;
    if (ok) {
        host.assign(params_ * (state ? 3 : 1), 0.0f);
        ok = std::fread(host.data(), sizeof(float), host.size(), f) == host.size() && std::fgetc(f) == EOF;
    }
    std::fclose(f);
    if (!ok) { error = std::string("not a denoiser checkpoint of this network: ") + path; return cudaErrorInvalidValue; }
    adamStep_ = state ? step : 0;
    cudaError_t e = cudaMemcpyAsync(master_, host.data(), sizeof(float) * params_, cudaMemcpyHostToDevice, stream_);
    if (state) {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(adamM_, host.data() + params_, sizeof(float) * params_, cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(adamV_, host.data() + 2 * params_, sizeof(float) * params_, cudaMemcpyHostToDevice, stream_);
    } else {
        if (e == cudaSuccess) e = cudaMemsetAsync(adamM_, 0, sizeof(float) * params_, stream_);
        if (e == cudaSuccess) e = cudaMemsetAsync(adamV_, 0, sizeof(float) * params_, stream_);
    }
    if (e == cudaSuccess) e = syncWeights(stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    return e;
}

}  // namespace rt
