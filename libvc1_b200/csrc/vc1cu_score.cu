// vc1cu_score.cu - candidate batch scoring, the VulkanComputeContext::score_motion_batch
// replacement (src/vulkan_compute.h:42-51, shader src/shaders/vulkan_motion_cost.comp).
//
// One warp per candidate: lanes stride over the block's sampled pixels (SAD) or 4x4 tiles
// (SATD), then a warp reduction. Two laws: the shader's (no legality gates, 32-bit
// accumulation) and the CPU's (block_sad_motion / mb_sad / block_satd_motion with the
// hidden-padding and odd-half-pel gates, encoder_motion.cpp:2197-3042).
#include <cuda_runtime.h>

#include "vc1cu_core.cuh"
#include "vc1cu_pred.cuh"

namespace vc1cu {

__global__ void score_kernel(const __grid_constant__ DevParams P, const __grid_constant__ ScoreArgs a, const int2* cands,
                             int n, unsigned long long* out) {
    const int lane = threadIdx.x & 31;
    const int ci = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    if (ci >= n) return;
    const int2 mv = cands[ci];
    const bool bil = mode_bilinear(a.mode);
    const GlobSampler gs{a.ref, a.pitch, a.W, a.H};
    const int aw = imax(0, imin(a.bw, a.W - a.x0)), ah = imax(0, imin(a.bh, a.H - a.y0));
    if (a.metric == VC1CU_METRIC_SAD) {
        bool bad = false;
        if (a.law == VC1CU_LAW_CPU) {
            if (a.stride > 1)
                bad = hidden_padding(P, a.x0, a.y0, 16, 16, mv.x, mv.y, VC1CU_MV_QPEL, true);
            else
                bad = hidden_padding(P, a.x0, a.y0, a.bw, a.bh, mv.x, mv.y, a.mode, chroma_gate(a.x0, a.y0, a.bw, a.bh)) ||
                      (bil && ((mv.x & 1) || (mv.y & 1)));
        }
        const int ss = imax(a.stride, 1);
        const int nsx = (aw + ss - 1) / ss, nsy = (ah + ss - 1) / ss;
        uint32_t part = 0;
        if (!bad)
            for (int i = lane; i < nsx * nsy; i += 32) {
                const int x = (i % nsx) * ss, y = (i / nsx) * ss;
                int pr[1];
                predict_row<1>(gs, bil, a.rnd, mv.x, mv.y, a.x0 + x, a.y0 + y, pr);
                part += (uint32_t)iabs((int)__ldg(a.cur + (size_t)(a.y0 + y) * a.pitch + a.x0 + x) - pr[0]);
            }
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) {
            if (bad) out[ci] = kBad;
            else if (a.law == VC1CU_LAW_SHADER) out[ci] = ss > 1 ? (uint32_t)(part * (uint32_t)(ss * ss)) : part;
            else out[ci] = ss > 1 ? (uint64_t)part * (uint64_t)(ss * ss) : (uint64_t)part;
        }
        return;
    }
    // SATD
    const bool bad = a.law == VC1CU_LAW_CPU && mode_halfpel(a.mode) && ((mv.x & 1) || (mv.y & 1));
    const int tx_n = (a.bw + 3) / 4, ty_n = (a.bh + 3) / 4;
    uint32_t part = 0;
    if (!bad)
        for (int t = lane; t < tx_n * ty_n; t += 32) {
            const int bx = (t % tx_n) * 4, by = (t / tx_n) * 4;
            if (!(bx < aw && by < ah)) continue;
            int d[16];
            for (int yy = 0; yy < 4; ++yy)
                for (int xx = 0; xx < 4; ++xx) {
                    const int px = bx + xx, py = by + yy;
                    int v = 0;
                    if (px < aw && py < ah) {
                        int pr[1];
                        predict_row<1>(gs, bil, a.rnd, mv.x, mv.y, a.x0 + px, a.y0 + py, pr);
                        v = (int)__ldg(a.cur + (size_t)(a.y0 + py) * a.pitch + a.x0 + px) - pr[0];
                    }
                    d[yy * 4 + xx] = v;
                }
            part += satd4x4(d);
        }
    for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) {
        if (a.law == VC1CU_LAW_CPU && (!aw || !ah)) out[ci] = 0;
        else out[ci] = bad ? kBad : (uint64_t)part;
    }
}

void launch_score(const DevParams& P, const ScoreArgs& a, const int2* cands, int n, unsigned long long* out,
                  cudaStream_t s) {
    const int warps_per_block = 8;
    score_kernel<<<(n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, s>>>(P, a, cands, n, out);
}

}  // namespace vc1cu

namespace vc1cu {

// INT32 lane-op throughput calibration: 8 independent chains of (add, xor) per thread, so
// every instruction is one 32-bit integer op with no dependency stall at full occupancy.
__global__ void int32_peak_kernel(uint32_t* out, int iters, uint32_t k1, uint32_t k2) {
    uint32_t a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = threadIdx.x * 2654435761u + (uint32_t)j * 40503u + blockIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            a[j] = a[j] + k1;
            a[j] = a[j] ^ k2;
        }
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) r ^= a[j];
    if (r == 0x9E3779B9u) out[0] = r;  // keeps the chains live
}

// Returns int32 lane-ops per second (16 ops per thread per iteration).
double measure_int32_peak(cudaStream_t s, int sms) {
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, 4) != cudaSuccess) return 0.0;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    int32_peak_kernel<<<blocks, threads, 0, s>>>(d, 64, 0x1234567u, 0x9abcdefu);  // warm-up
    cudaEventRecord(a, s);
    int32_peak_kernel<<<blocks, threads, 0, s>>>(d, iters, 0x1234567u, 0x9abcdefu);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (ms <= 0.f) return 0.0;
    return 16.0 * iters * (double)blocks * threads / (ms * 1e-3);
}

// FP64 throughput calibration: 8 independent chains of fused multiply-adds per thread (two
// flops each), contracting values that stay normal.
__global__ void fp64_peak_kernel(double* out, int iters, double k1, double k2) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = 1.0 + threadIdx.x * 1e-3 + j * 0.25 + blockIdx.x * 1e-6;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = __fma_rn(a[j], k1, k2);
    }
    double r = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) r += a[j];
    if (r == 1234.5) out[0] = r;  // keeps the chains live
}

// Returns FP64 flops per second (16 per thread per iteration).
double measure_fp64_peak(cudaStream_t s, int sms) {
    double* d = nullptr;
    if (cudaMalloc(&d, 8) != cudaSuccess) return 0.0;
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fp64_peak_kernel<<<blocks, threads, 0, s>>>(d, 256, 0.999999, 1e-7);  // warm-up
    cudaEventRecord(a, s);
    fp64_peak_kernel<<<blocks, threads, 0, s>>>(d, iters, 0.999999, 1e-7);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (ms <= 0.f) return 0.0;
    return 16.0 * iters * (double)blocks * threads / (ms * 1e-3);
}

}  // namespace vc1cu
