// lgm_probe.cu -- measured arithmetic peaks of the device the pair sums run on.
//
// The pair kernels are bounded by FP32 FMA issue and by the MUFU (SFU) pipe
// (rsqrt), not by HBM or the tensor cores.  These probes measure what one
// B200 sustains on each, with CUDA events, so that the roofline fractions of
// the pair kernels can be stated against a measured figure beside the one
// derived from the SM count and clock:
//   FFMA    scalar fmaf, 8 independent chains per thread;
//   FFMA2   packed FP32x2 fma (two lanes per instruction), 8 chains;
//   MUFU    rsqrt.approx.ftz.f32, 8 independent chains per thread.
// Every chain's result feeds a sum that is stored only under a condition the
// inputs never meet, so the compiler keeps every instruction.
#include <cuda_runtime.h>

#include "langmuir_b200.h"
#include "lgm_device.cuh"

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeBlocksPerSm = 8;
constexpr int kChains = 8;

__global__ void __launch_bounds__(kProbeThreads) probe_ffma(float* sink, int iters, float a,
                                                           float b) {
    float x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == -1.2345f) sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kProbeThreads) probe_ffma2(float* sink, int iters, float a,
                                                            float b) {
    float2 x[kChains];
    const float2 av = make_float2(a, a), bv = make_float2(b, b);
#pragma unroll
    for (int k = 0; k < kChains; ++k)
        x[k] = make_float2((float)(threadIdx.x + k) * 1e-3f, (float)(threadIdx.x - k) * 1e-3f);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = __ffma2_rn(x[k], av, bv);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k].x + x[k].y;
    if (s == -1.2345f) sink[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kProbeThreads) probe_rsqrt(float* sink, int iters) {
    float x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = 1.5f + (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = lgm::rsqrt_mufu(x[k]);  // stays near 1
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    if (s == -1.2345f) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" lgm_status lgm_probe_peaks(int32_t device, lgm_peaks* out) {
    if (!out) return LGM_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return LGM_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return LGM_ERR_CUDA;
    int sms = 0, clock_khz = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, device) != cudaSuccess)
        return LGM_ERR_CUDA;
    const int blocks = sms * kProbeBlocksPerSm;
    const double threads = (double)blocks * kProbeThreads;
    float* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaMalloc(&sink, sizeof(float) * blocks) != cudaSuccess) return LGM_ERR_CUDA;
    lgm_status st = LGM_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        st = LGM_ERR_CUDA;
    } else {
        // best of five launches of each probe after one warm-up launch
        auto time_best = [&](auto launch) -> float {
            launch();
            float best = 1e30f;
            for (int r = 0; r < 5; ++r) {
                cudaEventRecord(e0);
                launch();
                cudaEventRecord(e1);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) best = ms;
            }
            return best;
        };
        const int it_fma = 1 << 15, it_rsq = 1 << 12;
        const float t_fma = time_best([&] {
            probe_ffma<<<blocks, kProbeThreads>>>(sink, it_fma, 0.999f, 1e-4f);
        });
        const float t_fma2 = time_best([&] {
            probe_ffma2<<<blocks, kProbeThreads>>>(sink, it_fma, 0.999f, 1e-4f);
        });
        const float t_rsq = time_best([&] {
            probe_rsqrt<<<blocks, kProbeThreads>>>(sink, it_rsq);
        });
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
            st = LGM_ERR_CUDA;
        } else {
            const double fma_ops = threads * kChains * (double)it_fma;  // per lane
            out->ffma_tflops = 2.0 * fma_ops / (t_fma * 1e-3) / 1e12;
            out->ffma2_tflops = 2.0 * 2.0 * fma_ops / (t_fma2 * 1e-3) / 1e12;
            out->rsqrt_per_s = threads * kChains * (double)it_rsq / (t_rsq * 1e-3);
            out->sm_count = sms;
            out->clock_mhz_attribute = clock_khz / 1000.0;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    return st;
}

namespace {

// The failure path of the pair kernels, made to run: both stages of a
// two-stage bulk-copy pipeline are armed for a chunk's bytes, but no copy is
// issued, so the bounded wait runs out (limit tries), raises DEVERR_TIMEOUT
// and the CTA drains its (absent) copies before leaving -- the same device
// functions the pair kernels call.  Nothing waits without a bound.
__global__ void __launch_bounds__(128) selftest_wait_timeout(unsigned* err, int limit) {
    __shared__ __align__(8) uint64_t bars[2];
    if (threadIdx.x == 0) {
        lgm::mbar_init(&bars[0], 1);
        lgm::mbar_init(&bars[1], 1);
        lgm::fence_mbar_init();
        lgm::mbar_arrive_expect_tx(&bars[0], 5120u);
        lgm::mbar_arrive_expect_tx(&bars[1], 5120u);
    }
    __syncthreads();
    const bool mine = lgm::mbar_wait_bounded(&bars[0], 0u, err, limit);
    if (!__syncthreads_and(mine) && threadIdx.x == 0) lgm::mbar_drain_stages(bars, 0u, 2u, limit);
}

// The same for the warp-specialised kernels' ring of four stages: all four
// are armed, no copy comes, every target warp's bounded wait on stage 0 runs
// out and leaves as a warp (the warp-uniform vote of pair_items_culled_ws),
// and the producer thread waits (bounded) for the ring's four phases before
// leaving (mbar_drain_ring).
__global__ void __launch_bounds__(160) selftest_ring_timeout(unsigned* err, int limit) {
    constexpr int S = 4;
    __shared__ __align__(8) uint64_t full[S];
    const int warp = (int)threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            lgm::mbar_init(&full[i], 1);
        }
        lgm::fence_mbar_init();
        for (int i = 0; i < S; ++i) lgm::mbar_arrive_expect_tx(&full[i], 5184u);
    }
    __syncthreads();
    if (warp == 4) {  // the producer warp
        if ((threadIdx.x & 31) == 0) lgm::mbar_drain_ring(full, S, 0u, (uint32_t)S, limit);
        return;
    }
    if (!__all_sync(0xffffffffu, lgm::mbar_wait_bounded(&full[0], 0u, err, limit))) return;
    atomicOr(err, lgm::DEVERR_STATE);  // a stage that no copy filled completed
}

}  // namespace

extern "C" lgm_status lgm_selftest_timeout(int32_t device, int32_t wait_limit) {
    if (wait_limit < 1 || wait_limit > (1 << 20)) return LGM_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return LGM_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return LGM_ERR_CUDA;
    unsigned* d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(unsigned)) != cudaSuccess) return LGM_ERR_CUDA;
    lgm_status st = LGM_OK;
    unsigned h_err = 0;
    if (cudaMemset(d_err, 0, sizeof(unsigned)) != cudaSuccess) {
        st = LGM_ERR_CUDA;
    } else {
        // the two-stage pipeline, then the four-stage ring: each must report
        // the timeout and nothing else
        unsigned h_ring = 0;
        selftest_wait_timeout<<<2, 128>>>(d_err, wait_limit);
        bool ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
                  cudaMemcpy(&h_err, d_err, sizeof h_err, cudaMemcpyDeviceToHost) == cudaSuccess &&
                  cudaMemset(d_err, 0, sizeof(unsigned)) == cudaSuccess;
        if (ok) {
            selftest_ring_timeout<<<2, 160>>>(d_err, wait_limit);
            ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
                 cudaMemcpy(&h_ring, d_err, sizeof h_ring, cudaMemcpyDeviceToHost) == cudaSuccess;
        }
        if (!ok)
            st = LGM_ERR_CUDA;
        else if (h_err == lgm::DEVERR_TIMEOUT && h_ring == lgm::DEVERR_TIMEOUT)
            st = LGM_ERR_TIMEOUT;
        else
            st = LGM_ERR_STATE;
    }
    cudaFree(d_err);
    return st;
}
