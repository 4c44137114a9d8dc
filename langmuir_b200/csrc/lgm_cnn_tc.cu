// lgm_cnn_tc.cu -- the surrogate's 32 -> 32 channel 3x3 convolution on the
// 5th-generation tensor cores: TMA tensor loads, tcgen05.mma with accumulators
// in tensor memory, a two-stage pipeline.
//
// Implicit GEMM per 8x16 output tile: M = 128 pixels, N = 32 output channels,
// K = 9 taps x 32 input channels, issued as 18 UMMA instructions of
// M128 N32 K16 (BF16 operands, FP32 accumulation) by one thread.
//
// A operand (pixels x channels, K-major, 64-byte swizzle): the input patch of
// a tile (10 x 18 pixels with the halo) is loaded three times, shifted by
// kx = 0, 1, 2 columns, each as one TMA box of 32 channels x 16 x 10 pixels
// of the NHWC tensor at (0, x0 + kx - 1, y0 - 1, b):
//     xs[kx][py * 16 + pc] = x[y0 + py - 1][x0 + pc + kx - 1][0 .. 31]   (64-byte rows)
// The tensor map fills outside the image with zeros (the halo) and writes the
// rows in the 64-byte swizzle pattern (16-byte chunk index XOR bits 1-2 of the
// row), which the UMMA descriptor (layout SWIZZLE_64B) reads back.  Tap
// (ky, kx) is then the 128 consecutive rows from row 16 ky of copy kx --
// 8-row atoms of 512 bytes (SBO) -- and K step j (channels 16j .. 16j+15) is
// the same rows at byte offset 32 j.  No im2col copy is made.
// B operand (output channels x channels, K-major, no swizzle): the weights,
// staged once per CTA as ws[tap][c8][out channel][8 channels] (8 x 16-byte
// core matrices, SBO 128 bytes, LBO one 8-channel plane).
//
// Pipeline (three stages of patch buffers and of 32 TMEM columns), warp
// specialised: one thread of warp 8 issues the TMA loads and the MMAs; two
// groups of four warps run the epilogue of alternate tiles (warps 0-3 the
// even, 4-7 the odd ones; warp w reads TMEM lanes 32 (w % 4) ..): tcgen05.ld
// of the accumulators, bias, ReLU, stores, 2x2 pooling with warp shuffles.  Three pairs of mbarriers hand the stages
// over: "full" (the patch has landed), "done" (the MMAs have finished: the
// accumulators are ready and the patch buffer is free) and "empty" (the
// epilogue has read the accumulators: the TMEM stage is free).  While the
// epilogue warps finish tile k, the tensor core computes tile k+1 and TMA
// loads tiles k+2 and k+3; three stages cover the copy latency, which is
// longer than one tile's MMAs.
//
// Every wait is bounded: a timeout sets a flag that lgm_cnn_error reports;
// the CTA then waits (bounded) for its own copies and MMAs, frees its TMEM and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "langmuir_b200_cnn.h"
#include "lgm_device.cuh"

namespace {

using bf16 = __nv_bfloat16;
using lgm::smem_addr;

constexpr int TY = 8, TX = 16;                 // output tile
constexpr int EPI_THREADS = 256;               // epilogue warps 0-7: two groups of four, a
                                               // group per stage, one pixel (TMEM lane) per thread
constexpr int THREADS = EPI_THREADS + 32;      // + warp 8: issues the copies and the MMAs
constexpr int COUT = LGM_CNN_CHANNELS;         // 32
constexpr int CIN = LGM_CNN_CHANNELS;          // 32
constexpr int C8 = CIN / 8;                    // 16-byte channel groups
constexpr int PROWS = TY + 2;                  // patch rows
constexpr int XPIX = PROWS * TX;               // rows of one shifted copy (160)
constexpr uint32_t COPY_BYTES = XPIX * CIN * 2u;           // 10240: one TMA box
constexpr uint32_t STAGE_BYTES = 3u * COPY_BYTES;          // 30720: one tile's patch copies
constexpr int NST = 3;                                     // pipeline stages
constexpr uint32_t XS_BYTES = NST * STAGE_BYTES;
constexpr uint32_t WS_BYTES = 9u * C8 * COUT * 16u;        // 18432
constexpr uint32_t SMEM_BYTES = XS_BYTES + WS_BYTES + 128; // + mbarriers and TMEM slot
constexpr uint32_t TMEM_COLS = 128;                        // NST stages of 32 columns (power of 2)

// Instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(COUT >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start address, leading
// (K-direction) and stride (M/N-direction) byte offsets in 16-byte units,
// descriptor version 1 at bit 46.
// layout: 0 no swizzle, 4 the 64-byte swizzle (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout = 0) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)(layout & 7u) << 61);
}

// One TMA box of the 4-D NHWC tensor map into shared memory, completion
// counted on `bar` (no multicast).
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16(hi)) << 16);
}

__device__ unsigned g_tc_error = 0;  // DEVERR_* bits of the tensor-core conv

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait that returns false after a timeout (and records it).
__device__ __forceinline__ bool wait(uint64_t* bar, int use) {
    return lgm::mbar_wait_bounded(bar, (uint32_t)(use & 1), &g_tc_error);
}

// x (through the tensor map): [B,H,W,32] bf16; w: [32][288] bf16
// (k = (ky*3 + kx)*32 + c); act [B,H,W,32] and/or pooled [B,H/2,W/2,32].
// H % 8 == 0, W % 16 == 0.
__global__ void __launch_bounds__(THREADS)
conv3x3_fwd_tc(const __grid_constant__ CUtensorMap xmap, const bf16* __restrict__ w,
               const float* __restrict__ bias, bf16* __restrict__ act, bf16* __restrict__ pooled,
               int B, int H, int W, int relu) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* ws = smem + XS_BYTES;            // [9][C8][COUT][16 B]
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + XS_BYTES + WS_BYTES);  // [NST]
    uint64_t* done = full + NST;                                                // [NST]
    uint64_t* empty = full + 2 * NST;                                           // [NST]
    // 3 * NST mbarriers (72 bytes), then the TMEM address
    static_assert(3 * NST * 8 <= 96, "mbarriers overlap the TMEM slot");
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + XS_BYTES + WS_BYTES + 96);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = W / TX, tiles_y = H / TY;
    const int ntiles = B * tiles_x * tiles_y;
    const int n = ((int)blockIdx.x < ntiles) ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(tslot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < 2 * NST; ++i) lgm::mbar_init(&full[i], 1);       // full, done
        for (int i = 2 * NST; i < 3 * NST; ++i) lgm::mbar_init(&full[i], 4);  // empty: a lane per
                                                                              // warp of a group
        lgm::fence_mbar_init();
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&xmap)) : "memory");
    }
    // weights, once: ws[t][c8][o] = w[o][t*32 + 8*c8 .. +8]
    for (int i = tid; i < 9 * C8 * COUT; i += THREADS) {
        const int o = i % COUT, c8 = (i / COUT) % C8, t = i / (COUT * C8);
        *reinterpret_cast<uint4*>(ws + (size_t)i * 16) =
            *reinterpret_cast<const uint4*>(w + (size_t)o * 9 * CIN + t * CIN + c8 * 8);
    }
    lgm::fence_proxy_async_smem();  // generic-proxy writes -> the tensor core's reads
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t xs_a = smem_addr(smem), ws_a = smem_addr(ws);

    auto origin = [&](int k, int& b, int& y0, int& x0) {
        const int tile = (int)blockIdx.x + k * (int)gridDim.x;
        b = tile / (tiles_x * tiles_y);
        const int rem = tile % (tiles_x * tiles_y);
        y0 = (rem / tiles_x) * TY;
        x0 = (rem % tiles_x) * TX;
    };

    if (warp == EPI_THREADS / 32) {
        // ---- producer: TMA loads and MMAs, one thread ----
        if (lane == 0 && n > 0) {
            int tma_issued = 0, mma_issued = 0, mma_waited = 0;
            bool ok = true;
            auto issue_tma = [&](int k) {
                const int st = k % NST;
                int b, y0, x0;
                origin(k, b, y0, x0);
                lgm::mbar_arrive_expect_tx(&full[st], STAGE_BYTES);
#pragma unroll 1
                for (int kx = 0; kx < 3; ++kx)
                    tma_load_4d(xs_a + st * STAGE_BYTES + kx * COPY_BYTES, &xmap, 0, x0 + kx - 1,
                                y0 - 1, b, &full[st]);
                ++tma_issued;
            };
            for (int k = 0; k < NST && k < n; ++k) issue_tma(k);
            for (int k = 0; k < n && ok; ++k) {
                const int st = k % NST;
                // the patch has landed; the epilogue has released the TMEM stage (tile k-NST)
                ok = wait(&full[st], k / NST) && (k < NST || wait(&empty[st], (k - NST) / NST));
                if (!ok) break;
                fence_after_sync();
                const uint32_t xa = xs_a + st * STAGE_BYTES, d = tmem + (uint32_t)(st * 32);
#pragma unroll 1
                for (int t = 0; t < 9; ++t) {
                    const int ky = t / 3, kx = t % 3;
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        // A: rows 16 ky .. 16 ky + 127 of copy kx, channels 16j .. 16j+15
                        const uint64_t da =
                            smem_desc(xa + kx * COPY_BYTES + ky * TX * 64 + j * 32, 16, 512, 4);
                        // B: 32 output channels of tap t, the same 16 channels
                        const uint64_t db =
                            smem_desc(ws_a + (uint32_t)(((t * C8 + 2 * j) * COUT) * 16), COUT * 16, 128);
                        umma(d, da, db, (t | j) ? 1u : 0u);
                    }
                }
                umma_commit(&done[st]);
                ++mma_issued;
                // tile k-1's MMAs finished -> its patch buffer takes tile k-1+NST
                if (k >= 1 && k - 1 + NST < n) {
                    ok = wait(&done[(k - 1) % NST], (k - 1) / NST);
                    mma_waited = k;
                    if (ok) issue_tma(k - 1 + NST);
                }
            }
            // after a timeout: wait (bounded) for the MMAs and copies still in flight
            for (int k = mma_waited; k < mma_issued; ++k)
                for (int it = 0; it < lgm::kWaitLimit; ++it)
                    if (lgm::mbar_try_wait(&done[k % NST], (uint32_t)((k / NST) & 1))) break;
            for (int k = mma_issued; k < tma_issued; ++k)
                for (int it = 0; it < lgm::kWaitLimit; ++it)
                    if (lgm::mbar_try_wait(&full[k % NST], (uint32_t)((k / NST) & 1))) break;
        }
    } else {
        // ---- epilogue: group g = warp / 4 takes the tiles k = g, g + 2, ...
        // (stage k % NST); thread = pixel = TMEM lane 32 (warp % 4) + lane ----
        const int g = warp >> 2, wq = warp & 3;
        float bv[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) bv[c] = bias ? bias[c] : 0.f;
        for (int k = g; k < n; k += 2) {
            const int st = k % NST;
            if (!wait(&done[st], k / NST)) break;
            fence_after_sync();
            float v[32];
            tmem_ld32(tmem + (uint32_t)(st * 32) + ((uint32_t)(wq * 32) << 16), v);
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);  // this warp's TMEM lanes are read
            int b, y0, x0;
            origin(k, b, y0, x0);
            // this thread's pixel: tile row 2*wq + lane/16, column lane%16
            const int r = 2 * wq + (lane >> 4), c = lane & 15;
#pragma unroll
            for (int ch = 0; ch < 32; ++ch) {
                v[ch] += bv[ch];
                if (relu) v[ch] = fmaxf(v[ch], 0.f);
            }
            if (act) {
                uint4* dst =
                    reinterpret_cast<uint4*>(act + (((size_t)b * H + y0 + r) * W + x0 + c) * COUT);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    dst[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                        pack2(v[8 * q + 4], v[8 * q + 5]),
                                        pack2(v[8 * q + 6], v[8 * q + 7]));
            }
            if (pooled) {
                // (row 2w + row 2w+1) first, then the column pair: lanes 16 apart, then 1 apart
#pragma unroll
                for (int ch = 0; ch < 32; ++ch) v[ch] += __shfl_down_sync(0xffffffffu, v[ch], 16);
#pragma unroll
                for (int ch = 0; ch < 32; ++ch) v[ch] += __shfl_down_sync(0xffffffffu, v[ch], 1);
                if (lane < 16 && (lane & 1) == 0) {
                    const int H2 = H / 2, W2 = W / 2;
                    uint4* dst = reinterpret_cast<uint4*>(
                        pooled + (((size_t)b * H2 + y0 / 2 + wq) * W2 + x0 / 2 + lane / 2) * COUT);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        dst[q] = make_uint4(pack2(0.25f * v[8 * q], 0.25f * v[8 * q + 1]),
                                            pack2(0.25f * v[8 * q + 2], 0.25f * v[8 * q + 3]),
                                            pack2(0.25f * v[8 * q + 4], 0.25f * v[8 * q + 5]),
                                            pack2(0.25f * v[8 * q + 6], 0.25f * v[8 * q + 7]));
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
}

}  // namespace

extern "C" {

lgm_status lgm_cnn_conv3x3_fwd_tc(const void* x, const void* w, const float* bias, void* act,
                                  void* pooled, int32_t B, int32_t H, int32_t W, int32_t relu,
                                  void* stream) {
    if (!x || !w || B < 1 || H < TY || W < TX || H % TY || W % TX || (!act && !pooled) ||
        (pooled && (H % 2 || W % 2)))
        return LGM_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)x | (uintptr_t)w | (uintptr_t)act | (uintptr_t)pooled) & 15u)
        return LGM_ERR_INVALID_ARGUMENT;  // TMA base and 16-byte vector accesses
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static int cap = 0;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return LGM_ERR_CUDA;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if (!cap) {
        // the whole unified L1/shared memory as shared memory: the default carveout
        // is sized for one CTA of this footprint per SM
        if (cudaFuncSetAttribute(conv3x3_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_BYTES) != cudaSuccess ||
            cudaFuncSetAttribute(conv3x3_fwd_tc, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return LGM_ERR_CUDA;
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int smem_sm = 0;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv3x3_fwd_tc, THREADS,
                                                          SMEM_BYTES) != cudaSuccess)
            per_sm = 0;
        // at least what the shared memory holds (1 KB reserved per CTA); TMEM: 512 columns
        per_sm = std::max(per_sm, smem_sm / (int)(SMEM_BYTES + 1024));
        per_sm = std::max(1, std::min(per_sm, (int)(512 / TMEM_COLS)));
        cap = sms * per_sm;
    }
    // NHWC bf16 tensor, dimensions innermost first (channel, x, y, image); one
    // box = 32 channels x 16 x 10 pixels, 64-byte rows in the 64-byte swizzle
    CUtensorMap map;
    const cuuint64_t dims[4] = {(cuuint64_t)CIN, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)W * CIN * 2,
                                   (cuuint64_t)H * W * CIN * 2};
    const cuuint32_t box[4] = {(cuuint32_t)CIN, (cuuint32_t)TX, (cuuint32_t)PROWS, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    if (encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return LGM_ERR_CUDA;
    const int ntiles = B * (H / TY) * (W / TX);
    conv3x3_fwd_tc<<<std::min(ntiles, cap), THREADS, SMEM_BYTES, (cudaStream_t)stream>>>(
        map, (const bf16*)w, bias, (bf16*)act, (bf16*)pooled, B, H, W, relu);
    return cudaGetLastError() == cudaSuccess ? LGM_OK : LGM_ERR_CUDA;
}

lgm_status lgm_cnn_error(uint32_t* flags) {
    if (!flags) return LGM_ERR_INVALID_ARGUMENT;
    unsigned v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_error, sizeof v) != cudaSuccess ||
        cudaMemcpyToSymbol(g_tc_error, &zero, sizeof zero) != cudaSuccess)
        return LGM_ERR_CUDA;
    *flags = v;
    return v ? LGM_ERR_TIMEOUT : LGM_OK;
}

}  // extern "C"
