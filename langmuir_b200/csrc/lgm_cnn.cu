// lgm_cnn.cu -- BF16 tensor-core kernels of the morphology surrogate.
//
// The surrogate maps a donor/acceptor morphology to (current, efficiency).
// Network: 4 x [3x3 conv, 32 channels, bias, ReLU] with 2x2 average pooling
// after the first three, global average pooling, then 32 -> 64 -> 2 fully
// connected.  Activations are NHWC BF16, weights BF16 copies of FP32 masters,
// every product accumulates in FP32 on the tensor cores (mma.sync m16n8k16).
//
//   conv3x3_fwd   implicit GEMM: a CTA computes 8x16 output pixels x 32
//                 channels from an input patch and the weights staged in
//                 shared memory; bias, ReLU and the 2x2 pool run in the
//                 epilogue.  With flipped, transposed weights and the plain
//                 epilogue it is also the input-gradient (dgrad) kernel.
//   conv3x3_wgrad weight and bias gradients: dW[n][k] = sum_p dA[p][n] X_col[p][k],
//                 split over pixel tiles, FP32 partials added atomically.
//   gemm_small    C = A B (+ bias, ReLU) for the fully connected layers with
//                 arbitrary strides, forward and backward.
//   pool/relu/gap element-wise passes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <type_traits>

#include "langmuir_b200_cnn.h"

namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D = A (16x16 bf16, row) * B (16x8 bf16, col) + C, FP32 accumulate.
__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int TY = 8, TX = 16;       // output tile (pixels) of a conv CTA
constexpr int CONV_THREADS = 128;    // 4 warps, warp w: rows 2w, 2w+1 of the tile
constexpr int COUT = LGM_CNN_CHANNELS;

template <int CIN>
struct ConvShape {
    static constexpr int KPAD = CIN == 1 ? 16 : 9 * CIN;  // GEMM K (CIN = 1 padded)
    static constexpr int CPAD = CIN == 1 ? 2 : CIN + 8;   // patch channel stride (bank skew)
    static constexpr int WSTRIDE = KPAD + 8;              // weight row stride
    static constexpr size_t PATCH = (size_t)(TY + 2) * (TX + 2) * CPAD;
    static constexpr int OSTR = COUT + 8;                 // staged output pixel stride
    static constexpr size_t OTILE = (size_t)TY * TX * OSTR;        // full-resolution tile
    static constexpr size_t PTILE = (size_t)(TY / 2) * (TX / 2) * OSTR;  // pooled tile
    static constexpr size_t SMEM = (PATCH + (size_t)COUT * WSTRIDE + OTILE + PTILE) * sizeof(bf16);
};

// Input patch of one 8x16 tile with a one-pixel halo, zero outside the image:
// patch[(py*(TX+2) + px)*CPAD + c] = x[b][y0+py-1][x0+px-1][c].  CIN = 32 moves
// 16-byte vectors (8 channels); CIN = 1 single values.
template <int CIN>
__device__ __forceinline__ void load_patch(const bf16* __restrict__ x, bf16* patch, int b, int y0,
                                           int x0, int H, int W, int tid) {
    using S = ConvShape<CIN>;
    if constexpr (CIN == 1) {
        for (int i = tid; i < (TY + 2) * (TX + 2); i += CONV_THREADS) {
            const int px = i % (TX + 2), py = i / (TX + 2);
            const int yy = y0 + py - 1, xx = x0 + px - 1;
            bf16 v = __float2bfloat16(0.f);
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = x[((size_t)b * H + yy) * W + xx];
            patch[i * S::CPAD] = v;
        }
    } else {
        constexpr int V = CIN / 8;  // 16-byte vectors per pixel
        for (int i = tid; i < (TY + 2) * (TX + 2) * V; i += CONV_THREADS) {
            const int c8 = i % V, pix = i / V;
            const int px = pix % (TX + 2), py = pix / (TX + 2);
            const int yy = y0 + py - 1, xx = x0 + px - 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < H && xx >= 0 && xx < W)
                v = *reinterpret_cast<const uint4*>(x + (((size_t)b * H + yy) * W + xx) * CIN + c8 * 8);
            *reinterpret_cast<uint4*>(patch + pix * S::CPAD + c8 * 8) = v;
        }
    }
}

// The patch of the next tile, held in registers while the current tile
// computes (software pipelining of the global loads): load() issues the
// loads, store() writes them to shared memory at the next tile's start.
template <int CIN>
struct PatchPrefetch {
    static constexpr int V = CIN == 1 ? 1 : CIN / 8;  // values per pixel
    static constexpr int ITEMS = (TY + 2) * (TX + 2) * V;
    static constexpr int PER = (ITEMS + CONV_THREADS - 1) / CONV_THREADS;
    using T = typename std::conditional<CIN == 1, unsigned short, uint4>::type;
    T r[PER];

    __device__ __forceinline__ void load(const bf16* __restrict__ x, int b, int y0, int x0, int H,
                                         int W, int tid) {
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = tid + k * CONV_THREADS;
            const int c8 = i % V, pix = i / V;
            const int px = pix % (TX + 2), py = pix / (TX + 2);
            const int yy = y0 + py - 1, xx = x0 + px - 1;
            const bool in = i < ITEMS && yy >= 0 && yy < H && xx >= 0 && xx < W;
            const size_t off = (((size_t)b * H + (in ? yy : 0)) * W + (in ? xx : 0)) * CIN + c8 * 8;
            if constexpr (CIN == 1) {
                r[k] = in ? reinterpret_cast<const unsigned short*>(x)[off] : (unsigned short)0;
            } else {
                r[k] = in ? *reinterpret_cast<const uint4*>(x + off) : make_uint4(0u, 0u, 0u, 0u);
            }
        }
    }
    __device__ __forceinline__ void store(bf16* patch, int tid) const {
        using S = ConvShape<CIN>;
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int i = tid + k * CONV_THREADS;
            if (i >= ITEMS) break;
            const int c8 = i % V, pix = i / V;
            if constexpr (CIN == 1) {
                reinterpret_cast<unsigned short*>(patch)[pix * S::CPAD] = r[k];
            } else {
                *reinterpret_cast<uint4*>(patch + pix * S::CPAD + c8 * 8) = r[k];
            }
        }
    }
};

// x: [B,H,W,CIN]; w: [COUT][KPAD] (k = (ky*3 + kx)*CIN + c); act: [B,H,W,COUT]
// (optional); pooled: [B,H/2,W/2,COUT] (optional).  H % 8 == 0, W % 16 == 0.
// Persistent over tiles: the weights are staged once per CTA, each 8x16 tile's
// patch is staged with vector loads, and the epilogue stages the output tile
// in shared memory so that global stores are whole 16-byte vectors.
template <int CIN>
__global__ void __launch_bounds__(CONV_THREADS)
conv3x3_fwd(const bf16* __restrict__ x, const bf16* __restrict__ w, const float* __restrict__ bias,
            bf16* __restrict__ act, bf16* __restrict__ pooled, int B, int H, int W, int relu) {
    using S = ConvShape<CIN>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* patch = reinterpret_cast<bf16*>(smem_raw);
    bf16* ws = patch + S::PATCH;
    bf16* ost = ws + COUT * S::WSTRIDE;
    bf16* pst = ost + S::OTILE;
    const int tiles_x = W / TX;
    const int tiles_y = H / TY;
    const int ntiles = B * tiles_x * tiles_y;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const bf16 zero = __float2bfloat16(0.f);

    for (int i = tid; i < COUT * S::KPAD; i += CONV_THREADS)
        ws[(i / S::KPAD) * S::WSTRIDE + (i % S::KPAD)] = w[i];
    float bv[4][2];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        bv[n][0] = bias ? bias[n * 8 + 2 * t] : 0.f;
        bv[n][1] = bias ? bias[n * 8 + 2 * t + 1] : 0.f;
    }

    PatchPrefetch<CIN> pf;
    auto origin = [&](int tile, int& b, int& y0, int& x0) {
        b = tile / (tiles_x * tiles_y);
        const int rem = tile % (tiles_x * tiles_y);
        y0 = (rem / tiles_x) * TY;
        x0 = (rem % tiles_x) * TX;
    };
    if ((int)blockIdx.x < ntiles) {
        int b0, y00, x00;
        origin(blockIdx.x, b0, y00, x00);
        pf.load(x, b0, y00, x00, H, W, tid);
    }
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int b, y0, x0;
        origin(tile, b, y0, x0);
        __syncthreads();  // the previous tile is done with patch, ost and pst
        pf.store(patch, tid);
        __syncthreads();
        if (tile + (int)gridDim.x < ntiles) {  // next tile's loads overlap this tile's math
            int bn, yn, xn;
            origin(tile + gridDim.x, bn, yn, xn);
            pf.load(x, bn, yn, xn, H, W, tid);
        }

        float acc[2][4][4];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int n = 0; n < 4; ++n)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][n][j] = 0.f;

        if constexpr (CIN == 1) {
            // one k16 step: the thread's columns k = 2t, 2t+1, 2t+8, 2t+9 are
            // taps (ky, kx) = (k / 3, k % 3) for k < 9 and zero padding above
            uint32_t bb[4][2];
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                const bf16* wr = ws + (n * 8 + g) * S::WSTRIDE;
                bb[n][0] = pack2(wr[2 * t], wr[2 * t + 1]);
                bb[n][1] = pack2(wr[2 * t + 8], wr[2 * t + 9]);
            }
            int toff[4];
            bool tok[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = 2 * t + (j & 1) + (j >> 1) * 8;
                tok[j] = k < 9;
                toff[j] = tok[j] ? ((k / 3) * (TX + 2) + k % 3) * S::CPAD : 0;
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = 2 * warp + i;
                const bf16* p0 = patch + (row * (TX + 2) + g) * S::CPAD;
                const bf16* p1 = p0 + 8 * S::CPAD;
                bf16 v0[4], v1[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    v0[j] = tok[j] ? p0[toff[j]] : zero;
                    v1[j] = tok[j] ? p1[toff[j]] : zero;
                }
                uint32_t a[4];
                a[0] = pack2(v0[0], v0[1]);
                a[1] = pack2(v1[0], v1[1]);
                a[2] = pack2(v0[2], v0[3]);
                a[3] = pack2(v1[2], v1[3]);
#pragma unroll
                for (int n = 0; n < 4; ++n) mma16816(acc[i][n], a, bb[n]);
            }
        } else {
#pragma unroll 2
            for (int s = 0; s < 9 * CIN / 16; ++s) {
                const int tap = (s * 16) / CIN, c0 = (s * 16) % CIN;
                const int ky = tap / 3, kx = tap % 3;
                uint32_t bb[4][2];
#pragma unroll
                for (int n = 0; n < 4; ++n) {
                    const bf16* wr = ws + (n * 8 + g) * S::WSTRIDE + s * 16;
                    bb[n][0] = *reinterpret_cast<const uint32_t*>(wr + 2 * t);
                    bb[n][1] = *reinterpret_cast<const uint32_t*>(wr + 2 * t + 8);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int row = 2 * warp + i + ky;
                    const bf16* p0 = patch + (row * (TX + 2) + g + kx) * S::CPAD + c0;
                    const bf16* p1 = patch + (row * (TX + 2) + g + 8 + kx) * S::CPAD + c0;
                    uint32_t a[4];
                    a[0] = *reinterpret_cast<const uint32_t*>(p0 + 2 * t);
                    a[1] = *reinterpret_cast<const uint32_t*>(p1 + 2 * t);
                    a[2] = *reinterpret_cast<const uint32_t*>(p0 + 2 * t + 8);
                    a[3] = *reinterpret_cast<const uint32_t*>(p1 + 2 * t + 8);
#pragma unroll
                    for (int n = 0; n < 4; ++n) mma16816(acc[i][n], a, bb[n]);
                }
            }
        }

        // epilogue: rows g / g+8 of the fragment are pixels x0+g / x0+g+8 of
        // tile row 2*warp+i; columns 2t, 2t+1 of n-tile n are channels n*8+2t, +1
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int ch = n * 8 + 2 * t;
            float v[2][4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                v[i][0] = acc[i][n][0] + bv[n][0];
                v[i][1] = acc[i][n][1] + bv[n][1];
                v[i][2] = acc[i][n][2] + bv[n][0];
                v[i][3] = acc[i][n][3] + bv[n][1];
                if (relu)
#pragma unroll
                    for (int j = 0; j < 4; ++j) v[i][j] = fmaxf(v[i][j], 0.f);
                if (act) {
                    const int r = 2 * warp + i;
                    *reinterpret_cast<uint32_t*>(ost + (r * TX + g) * S::OSTR + ch) =
                        pack2(__float2bfloat16(v[i][0]), __float2bfloat16(v[i][1]));
                    *reinterpret_cast<uint32_t*>(ost + (r * TX + g + 8) * S::OSTR + ch) =
                        pack2(__float2bfloat16(v[i][2]), __float2bfloat16(v[i][3]));
                }
            }
            if (pooled) {
                // sum the two tile rows (same thread), then the x pair (lanes g, g^1)
                float sm[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) sm[j] = v[0][j] + v[1][j];
#pragma unroll
                for (int j = 0; j < 4; ++j) sm[j] += __shfl_xor_sync(0xffffffffu, sm[j], 4);
                if ((g & 1) == 0) {
                    // pooled tile: row warp (0..3), columns g/2 and g/2 + 4 (0..7)
                    *reinterpret_cast<uint32_t*>(pst + (warp * (TX / 2) + g / 2) * S::OSTR + ch) =
                        pack2(__float2bfloat16(0.25f * sm[0]), __float2bfloat16(0.25f * sm[1]));
                    *reinterpret_cast<uint32_t*>(pst + (warp * (TX / 2) + g / 2 + 4) * S::OSTR + ch) =
                        pack2(__float2bfloat16(0.25f * sm[2]), __float2bfloat16(0.25f * sm[3]));
                }
            }
        }
        __syncthreads();
        constexpr int VO = COUT / 8;  // 16-byte vectors per output pixel
        if (act) {
            for (int i = tid; i < TY * TX * VO; i += CONV_THREADS) {
                const int c8 = i % VO, pix = i / VO;
                const int r = pix / TX, c = pix % TX;
                *reinterpret_cast<uint4*>(act + (((size_t)b * H + y0 + r) * W + x0 + c) * COUT + c8 * 8) =
                    *reinterpret_cast<const uint4*>(ost + pix * S::OSTR + c8 * 8);
            }
        }
        if (pooled) {
            const int H2 = H / 2, W2 = W / 2;
            for (int i = tid; i < (TY / 2) * (TX / 2) * VO; i += CONV_THREADS) {
                const int c8 = i % VO, pix = i / VO;
                const int r = pix / (TX / 2), c = pix % (TX / 2);
                *reinterpret_cast<uint4*>(
                    pooled + (((size_t)b * H2 + y0 / 2 + r) * W2 + x0 / 2 + c) * COUT + c8 * 8) =
                    *reinterpret_cast<const uint4*>(pst + pix * S::OSTR + c8 * 8);
            }
        }
    }
}

// The first layer (one input channel) on a wide tile.  With 9 taps the GEMM
// is one k16 step per 16 pixels, so the 8x16 tile of conv3x3_fwd spends its
// time in barriers and staging; here a CTA takes 8 rows x 64 pixels per
// iteration (4 sub-tiles of 16 per warp row pair), with one patch, one set of
// barriers and one vectorised store of the tile.  Same arithmetic and layouts
// as conv3x3_fwd<1>: x [B,H,W] bf16, w [COUT][16] (taps 0..8, zero padding),
// act [B,H,W,COUT] and pooled [B,H/2,W/2,COUT], each optional.
constexpr int C1_TX = 64;                               // tile width of the first layer
constexpr int C1_CPAD = 2;                              // patch pixel stride (bf16)
constexpr int C1_PATCH = (TY + 2) * (C1_TX + 2);        // patch pixels
constexpr int C1_WSTRIDE = 16 + 8;
constexpr int C1_OSTR = COUT + 8;
constexpr int C1_PER = (C1_PATCH + CONV_THREADS - 1) / CONV_THREADS;
constexpr size_t C1_SMEM_BASE =
    ((size_t)C1_PATCH * C1_CPAD + (size_t)COUT * C1_WSTRIDE + (size_t)(TY / 2) * (C1_TX / 2) * C1_OSTR) *
    sizeof(bf16);
constexpr size_t C1_SMEM_ACT = (size_t)TY * C1_TX * C1_OSTR * sizeof(bf16);

__global__ void __launch_bounds__(CONV_THREADS)
conv1_fwd(const bf16* __restrict__ x, const bf16* __restrict__ w, const float* __restrict__ bias,
          bf16* __restrict__ act, bf16* __restrict__ pooled, int B, int H, int W, int relu) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* patch = reinterpret_cast<bf16*>(smem_raw);
    bf16* ws = patch + C1_PATCH * C1_CPAD;
    bf16* pst = ws + COUT * C1_WSTRIDE;                   // [(TY/2)*(C1_TX/2)][C1_OSTR]
    bf16* ost = pst + (TY / 2) * (C1_TX / 2) * C1_OSTR;   // [TY*C1_TX][C1_OSTR], if act
    const int tiles_x = W / C1_TX, tiles_y = H / TY;
    const int ntiles = B * tiles_x * tiles_y;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const bf16 zero = __float2bfloat16(0.f);

    for (int i = tid; i < COUT * 16; i += CONV_THREADS) ws[(i / 16) * C1_WSTRIDE + (i % 16)] = w[i];
    float bv[4][2];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        bv[n][0] = bias ? bias[n * 8 + 2 * t] : 0.f;
        bv[n][1] = bias ? bias[n * 8 + 2 * t + 1] : 0.f;
    }
    __syncthreads();
    // the thread's B fragments and tap offsets: columns k = 2t, 2t+1, 2t+8, 2t+9
    // are taps (ky, kx) = (k / 3, k % 3) for k < 9, zero padding above
    uint32_t bb[4][2];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const bf16* wr = ws + (n * 8 + g) * C1_WSTRIDE;
        bb[n][0] = pack2(wr[2 * t], wr[2 * t + 1]);
        bb[n][1] = pack2(wr[2 * t + 8], wr[2 * t + 9]);
    }
    int toff[4];
    bool tok[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int k = 2 * t + (j & 1) + (j >> 1) * 8;
        tok[j] = k < 9;
        toff[j] = tok[j] ? ((k / 3) * (C1_TX + 2) + k % 3) * C1_CPAD : 0;
    }

    unsigned short pre[C1_PER];
    auto origin = [&](int tile, int& b, int& y0, int& x0) {
        b = tile / (tiles_x * tiles_y);
        const int rem = tile % (tiles_x * tiles_y);
        y0 = (rem / tiles_x) * TY;
        x0 = (rem % tiles_x) * C1_TX;
    };
    auto prefetch = [&](int tile) {
        int b, y0, x0;
        origin(tile, b, y0, x0);
#pragma unroll
        for (int k = 0; k < C1_PER; ++k) {
            const int i = tid + k * CONV_THREADS;
            const int px = i % (C1_TX + 2), py = i / (C1_TX + 2);
            const int yy = y0 + py - 1, xx = x0 + px - 1;
            const bool in = i < C1_PATCH && yy >= 0 && yy < H && xx >= 0 && xx < W;
            pre[k] = in ? reinterpret_cast<const unsigned short*>(x)[((size_t)b * H + yy) * W + xx]
                        : (unsigned short)0;
        }
    };
    if ((int)blockIdx.x < ntiles) prefetch(blockIdx.x);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int b, y0, x0;
        origin(tile, b, y0, x0);
        __syncthreads();  // the previous tile is done with patch, ost and pst
#pragma unroll
        for (int k = 0; k < C1_PER; ++k) {
            const int i = tid + k * CONV_THREADS;
            if (i < C1_PATCH) reinterpret_cast<unsigned short*>(patch)[i * C1_CPAD] = pre[k];
        }
        __syncthreads();
        if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x);  // overlaps the math

#pragma unroll
        for (int sx = 0; sx < C1_TX / TX; ++sx) {
            float acc[2][4][4];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int n = 0; n < 4; ++n)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][n][j] = 0.f;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = 2 * warp + i;
                const bf16* p0 = patch + (row * (C1_TX + 2) + sx * TX + g) * C1_CPAD;
                const bf16* p1 = p0 + 8 * C1_CPAD;
                bf16 v0[4], v1[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    v0[j] = tok[j] ? p0[toff[j]] : zero;
                    v1[j] = tok[j] ? p1[toff[j]] : zero;
                }
                uint32_t a[4];
                a[0] = pack2(v0[0], v0[1]);
                a[1] = pack2(v1[0], v1[1]);
                a[2] = pack2(v0[2], v0[3]);
                a[3] = pack2(v1[2], v1[3]);
#pragma unroll
                for (int n = 0; n < 4; ++n) mma16816(acc[i][n], a, bb[n]);
            }
            // epilogue of the sub-tile: rows g / g+8 of a fragment are pixels
            // sx*16 + g / + 8 of tile row 2*warp + i; columns 2t, 2t+1 of n-tile
            // n are channels n*8 + 2t, + 1
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                const int ch = n * 8 + 2 * t;
                float v[2][4];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    v[i][0] = acc[i][n][0] + bv[n][0];
                    v[i][1] = acc[i][n][1] + bv[n][1];
                    v[i][2] = acc[i][n][2] + bv[n][0];
                    v[i][3] = acc[i][n][3] + bv[n][1];
                    if (relu)
#pragma unroll
                        for (int j = 0; j < 4; ++j) v[i][j] = fmaxf(v[i][j], 0.f);
                    if (act) {
                        const int r = 2 * warp + i, c = sx * TX + g;
                        *reinterpret_cast<uint32_t*>(ost + (r * C1_TX + c) * C1_OSTR + ch) =
                            pack2(__float2bfloat16(v[i][0]), __float2bfloat16(v[i][1]));
                        *reinterpret_cast<uint32_t*>(ost + (r * C1_TX + c + 8) * C1_OSTR + ch) =
                            pack2(__float2bfloat16(v[i][2]), __float2bfloat16(v[i][3]));
                    }
                }
                if (pooled) {
                    float sm[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) sm[j] = v[0][j] + v[1][j];
#pragma unroll
                    for (int j = 0; j < 4; ++j) sm[j] += __shfl_xor_sync(0xffffffffu, sm[j], 4);
                    if ((g & 1) == 0) {
                        // pooled row warp, columns sx*8 + g/2 and sx*8 + g/2 + 4
                        const int pc = sx * (TX / 2) + g / 2;
                        *reinterpret_cast<uint32_t*>(pst + (warp * (C1_TX / 2) + pc) * C1_OSTR + ch) =
                            pack2(__float2bfloat16(0.25f * sm[0]), __float2bfloat16(0.25f * sm[1]));
                        *reinterpret_cast<uint32_t*>(pst + (warp * (C1_TX / 2) + pc + 4) * C1_OSTR + ch) =
                            pack2(__float2bfloat16(0.25f * sm[2]), __float2bfloat16(0.25f * sm[3]));
                    }
                }
            }
        }
        __syncthreads();
        constexpr int VO = COUT / 8;  // 16-byte vectors per output pixel
        if (act) {
            for (int i = tid; i < TY * C1_TX * VO; i += CONV_THREADS) {
                const int c8 = i % VO, pix = i / VO;
                const int r = pix / C1_TX, c = pix % C1_TX;
                *reinterpret_cast<uint4*>(act + (((size_t)b * H + y0 + r) * W + x0 + c) * COUT + c8 * 8) =
                    *reinterpret_cast<const uint4*>(ost + pix * C1_OSTR + c8 * 8);
            }
        }
        if (pooled) {
            const int H2 = H / 2, W2 = W / 2;
            for (int i = tid; i < (TY / 2) * (C1_TX / 2) * VO; i += CONV_THREADS) {
                const int c8 = i % VO, pix = i / VO;
                const int r = pix / (C1_TX / 2), c = pix % (C1_TX / 2);
                *reinterpret_cast<uint4*>(
                    pooled + (((size_t)b * H2 + y0 / 2 + r) * W2 + x0 / 2 + c) * COUT + c8 * 8) =
                    *reinterpret_cast<const uint4*>(pst + pix * C1_OSTR + c8 * 8);
            }
        }
    }
}

// Weight/bias gradients.  GEMM with M = COUT (2 m16 tiles), N = KPAD,
// K = pixels: A(n, p) = dA[p][n], B(p, k) = x_col[p][k].  A CTA walks pixel
// tiles of 8x16 with a grid stride, keeps its partial dW in registers and
// adds it to dW once.  Warp w owns n-tiles w, w+4, ... of the NT n-tiles.
template <int CIN>
__global__ void __launch_bounds__(CONV_THREADS)
conv3x3_wgrad(const bf16* __restrict__ x, const bf16* __restrict__ dA, float* __restrict__ dW,
              float* __restrict__ db, int B, int H, int W) {
    using S = ConvShape<CIN>;
    constexpr int NT = S::KPAD / 8;                 // n8 tiles (36 or 2)
    constexpr int NTW = (NT + 3) / 4;               // per warp
    constexpr int DSTR = COUT + 8;                  // dA tile row stride
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* patch = reinterpret_cast<bf16*>(smem_raw);
    bf16* dtile = patch + S::PATCH;                 // [TY*TX][DSTR]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const int tiles_x = W / TX, tiles_y = H / TY;
    const int ntiles = B * tiles_x * tiles_y;
    float acc[2][NTW][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int n = 0; n < NTW; ++n)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][n][j] = 0.f;
    float bsum = 0.f;  // bias gradient: thread tid < COUT sums channel tid
    const bf16 zero = __float2bfloat16(0.f);

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = tile / (tiles_x * tiles_y);
        const int rem = tile % (tiles_x * tiles_y);
        const int y0 = (rem / tiles_x) * TY, x0 = (rem % tiles_x) * TX;
        __syncthreads();
        load_patch<CIN>(x, patch, b, y0, x0, H, W, tid);
        for (int i = tid; i < TY * TX * (COUT / 8); i += CONV_THREADS) {
            const int c8 = i % (COUT / 8), p = i / (COUT / 8);
            const int yy = y0 + p / TX, xx = x0 + p % TX;
            *reinterpret_cast<uint4*>(dtile + p * DSTR + c8 * 8) =
                *reinterpret_cast<const uint4*>(dA + (((size_t)b * H + yy) * W + xx) * COUT + c8 * 8);
        }
        __syncthreads();
        if (tid < COUT)
            for (int p = 0; p < TY * TX; ++p) bsum += __bfloat162float(dtile[p * DSTR + tid]);
        // K loop over the tile's 128 pixels in k16 steps
#pragma unroll 1
        for (int ks = 0; ks < TY * TX / 16; ++ks) {
            const int p0 = ks * 16;
            uint32_t a[2][4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int n0 = i * 16 + g, n1 = n0 + 8;
                const int pa = p0 + 2 * t, pb = p0 + 2 * t + 8;
                a[i][0] = pack2(dtile[pa * DSTR + n0], dtile[(pa + 1) * DSTR + n0]);
                a[i][1] = pack2(dtile[pa * DSTR + n1], dtile[(pa + 1) * DSTR + n1]);
                a[i][2] = pack2(dtile[pb * DSTR + n0], dtile[(pb + 1) * DSTR + n0]);
                a[i][3] = pack2(dtile[pb * DSTR + n1], dtile[(pb + 1) * DSTR + n1]);
            }
            // B(p, k): pixel p of the tile, k = (ky*3 + kx)*CIN + c
            auto xcol = [&](int p, int k) -> bf16 {
                if (k >= 9 * CIN) return zero;
                const int tapk = k / CIN, c = k % CIN;
                const int py = p / TX + tapk / 3, px = p % TX + tapk % 3;
                return patch[(py * (TX + 2) + px) * S::CPAD + c];
            };
#pragma unroll
            for (int nn = 0; nn < NTW; ++nn) {
                const int nt = warp + 4 * nn;
                if (nt >= NT) break;
                const int k = nt * 8 + g;
                const int pa = p0 + 2 * t, pb = p0 + 2 * t + 8;
                uint32_t bb[2];
                bb[0] = pack2(xcol(pa, k), xcol(pa + 1, k));
                bb[1] = pack2(xcol(pb, k), xcol(pb + 1, k));
                mma16816(acc[0][nn], a[0], bb);
                mma16816(acc[1][nn], a[1], bb);
            }
        }
    }
    // C tile (m16 x n8): rows g, g+8 -> out channel; cols 2t, 2t+1 -> k
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int nn = 0; nn < NTW; ++nn) {
            const int nt = warp + 4 * nn;
            if (nt >= NT) break;
            const int k = nt * 8 + 2 * t;
            const int n0 = i * 16 + g, n1 = n0 + 8;
            atomicAdd(&dW[n0 * S::KPAD + k], acc[i][nn][0]);
            atomicAdd(&dW[n0 * S::KPAD + k + 1], acc[i][nn][1]);
            atomicAdd(&dW[n1 * S::KPAD + k], acc[i][nn][2]);
            atomicAdd(&dW[n1 * S::KPAD + k + 1], acc[i][nn][3]);
        }
    if (tid < COUT && db) atomicAdd(&db[tid], bsum);
}

// C[M][N] (fp32, row stride N) = sum_k A(m, k) B(k, n) (+ bias[n], ReLU),
// A(m, k) = A[m*sam + k*sak], B(k, n) = B[k*sbk + n*sbn]; out of range -> 0.
// accumulate != 0: C += result (atomic).  One warp per 16x8 output tile.
__global__ void gemm_small(const bf16* __restrict__ A, int sam, int sak, const bf16* __restrict__ Bm,
                          int sbk, int sbn, float* __restrict__ C, const float* __restrict__ bias,
                          int M, int N, int K, int relu, int accumulate) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int mt = (M + 15) / 16, nt = (N + 7) / 8;
    if (warp >= mt * nt) return;
    const int m0 = (warp / nt) * 16, n0 = (warp % nt) * 8;
    const bf16 zero = __float2bfloat16(0.f);
    auto a_at = [&](int m, int k) { return (m < M && k < K) ? A[(size_t)m * sam + (size_t)k * sak] : zero; };
    auto b_at = [&](int k, int n) { return (k < K && n < N) ? Bm[(size_t)k * sbk + (size_t)n * sbn] : zero; };
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[4], b[2];
        a[0] = pack2(a_at(m0 + g, k0 + 2 * t), a_at(m0 + g, k0 + 2 * t + 1));
        a[1] = pack2(a_at(m0 + g + 8, k0 + 2 * t), a_at(m0 + g + 8, k0 + 2 * t + 1));
        a[2] = pack2(a_at(m0 + g, k0 + 2 * t + 8), a_at(m0 + g, k0 + 2 * t + 9));
        a[3] = pack2(a_at(m0 + g + 8, k0 + 2 * t + 8), a_at(m0 + g + 8, k0 + 2 * t + 9));
        b[0] = pack2(b_at(k0 + 2 * t, n0 + g), b_at(k0 + 2 * t + 1, n0 + g));
        b[1] = pack2(b_at(k0 + 2 * t + 8, n0 + g), b_at(k0 + 2 * t + 9, n0 + g));
        mma16816(c, a, b);
    }
    const int rows[2] = {m0 + g, m0 + g + 8};
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int m = rows[r], n = n0 + 2 * t + j;
            if (m >= M || n >= N) continue;
            float v = c[2 * r + j] + (bias ? bias[n] : 0.f);
            if (relu) v = fmaxf(v, 0.f);
            if (accumulate) atomicAdd(&C[(size_t)m * N + n], v);
            else C[(size_t)m * N + n] = v;
        }
}

// dA_pre = (act > 0) * (pooled-grad / 4 or full-grad), pooled: [B,H/2,W/2,C].
__global__ void relu_pool_bwd(const bf16* __restrict__ act, const bf16* __restrict__ dP,
                              bf16* __restrict__ dA, int B, int H, int W, int pooled) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)B * H * W * COUT;
    if (i >= n) return;
    const int c = (int)(i % COUT);
    const size_t pix = i / COUT;
    const int xx = (int)(pix % W), yy = (int)((pix / W) % H), b = (int)(pix / ((size_t)W * H));
    float g;
    if (pooled) {
        const int H2 = H / 2, W2 = W / 2;
        g = 0.25f * __bfloat162float(dP[(((size_t)b * H2 + yy / 2) * W2 + xx / 2) * COUT + c]);
    } else {
        g = __bfloat162float(dP[i]);
    }
    dA[i] = __float2bfloat16(__bfloat162float(act[i]) > 0.f ? g : 0.f);
}

// global average pool: g[b][c] = mean over pixels (fp32 and bf16 copies)
__global__ void gap_fwd(const bf16* __restrict__ act, float* __restrict__ out32,
                        bf16* __restrict__ out16, int HW) {
    const int b = blockIdx.x, c = threadIdx.x;  // blockDim = COUT
    float s = 0.f;
    for (int p = 0; p < HW; ++p) s += __bfloat162float(act[((size_t)b * HW + p) * COUT + c]);
    s /= (float)HW;
    out32[b * COUT + c] = s;
    out16[b * COUT + c] = __float2bfloat16(s);
}

// d act = (act > 0) * dg[b][c] / HW
__global__ void gap_relu_bwd(const bf16* __restrict__ act, const float* __restrict__ dg,
                             bf16* __restrict__ dA, int B, int HW) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)B * HW * COUT) return;
    const int c = (int)(i % COUT), b = (int)(i / ((size_t)HW * COUT));
    const float g = dg[b * COUT + c] / (float)HW;
    dA[i] = __float2bfloat16(__bfloat162float(act[i]) > 0.f ? g : 0.f);
}

__global__ void f32_to_bf16(const float* __restrict__ in, bf16* __restrict__ out, int n, int relu_mask_from,
                            const float* __restrict__ mask_src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = in[i];
    if (relu_mask_from && mask_src && mask_src[i] <= 0.f) v = 0.f;
    out[i] = __float2bfloat16(v);
}

// dgrad weights: wd[c][(ky*3+kx)*COUT + o] = w[o][((2-ky)*3 + (2-kx))*CIN + c]
__global__ void flip_weights(const bf16* __restrict__ w, bf16* __restrict__ wd, int cin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cin * 9 * COUT) return;
    const int o = i % COUT, tap = (i / COUT) % 9, c = i / (9 * COUT);
    wd[i] = w[o * 9 * cin + (8 - tap) * cin + c];
}

lgm_status launch_check() {
    return cudaGetLastError() == cudaSuccess ? LGM_OK : LGM_ERR_CUDA;
}

}  // namespace

extern "C" {

lgm_status lgm_cnn_conv3x3_fwd(int32_t cin, const void* x, const void* w, const float* bias,
                               void* act, void* pooled, int32_t B, int32_t H, int32_t W,
                               int32_t relu, void* stream) {
    if ((cin != 1 && cin != LGM_CNN_CHANNELS) || !x || !w || B < 1 || H % TY || W % TX ||
        (pooled && (H % 2 || W % 2)) || (!act && !pooled))
        return LGM_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    if (cin == 1 && W % C1_TX == 0) {
        // the wide-tile first layer; persistent: at most the CTAs resident at once
        const size_t smem = C1_SMEM_BASE + (act ? C1_SMEM_ACT : 0);
        static int cap1[2] = {0, 0};
        const int ai = act ? 1 : 0;
        if (!cap1[ai]) {
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaFuncSetAttribute(conv1_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(C1_SMEM_BASE + C1_SMEM_ACT));
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv1_fwd, CONV_THREADS, smem);
            cap1[ai] = std::max(1, sms * std::max(1, per_sm));
        }
        const int ntiles1 = B * (H / TY) * (W / C1_TX);
        conv1_fwd<<<std::min(ntiles1, cap1[ai]), CONV_THREADS, smem, st>>>(
            (const bf16*)x, (const bf16*)w, bias, (bf16*)act, (bf16*)pooled, B, H, W, relu);
        return launch_check();
    }
    const int ntiles = B * (H / TY) * (W / TX);
    // persistent: at most the CTAs that fit on the device at once
    static int cap[2] = {0, 0};
    const int ci = cin == 1 ? 0 : 1;
    if (!cap[ci]) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (ci == 0)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv3x3_fwd<1>, CONV_THREADS,
                                                          ConvShape<1>::SMEM);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conv3x3_fwd<COUT>, CONV_THREADS,
                                                          ConvShape<COUT>::SMEM);
        cap[ci] = std::max(1, sms * std::max(1, per_sm));
    }
    const int grid = std::min(ntiles, cap[ci]);
    if (cin == 1) {
        conv3x3_fwd<1><<<grid, CONV_THREADS, ConvShape<1>::SMEM, st>>>(
            (const bf16*)x, (const bf16*)w, bias, (bf16*)act, (bf16*)pooled, B, H, W, relu);
    } else {
        conv3x3_fwd<COUT><<<grid, CONV_THREADS, ConvShape<COUT>::SMEM, st>>>(
            (const bf16*)x, (const bf16*)w, bias, (bf16*)act, (bf16*)pooled, B, H, W, relu);
    }
    return launch_check();
}

lgm_status lgm_cnn_conv3x3_wgrad(int32_t cin, const void* x, const void* dA, float* dW, float* db,
                                 int32_t B, int32_t H, int32_t W, void* stream) {
    if ((cin != 1 && cin != LGM_CNN_CHANNELS) || !x || !dA || !dW || B < 1 || H % TY || W % TX)
        return LGM_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    const int tiles = B * (H / TY) * (W / TX);
    const int grid = tiles < 148 * 4 ? tiles : 148 * 4;
    constexpr size_t dsz = (size_t)TY * TX * (COUT + 8) * sizeof(bf16);
    if (cin == 1) {
        conv3x3_wgrad<1><<<grid, CONV_THREADS, ConvShape<1>::PATCH * sizeof(bf16) + dsz, st>>>(
            (const bf16*)x, (const bf16*)dA, dW, db, B, H, W);
    } else {
        conv3x3_wgrad<COUT><<<grid, CONV_THREADS, ConvShape<COUT>::PATCH * sizeof(bf16) + dsz, st>>>(
            (const bf16*)x, (const bf16*)dA, dW, db, B, H, W);
    }
    return launch_check();
}

lgm_status lgm_cnn_flip_weights(int32_t cin, const void* w, void* wd, void* stream) {
    if (cin != LGM_CNN_CHANNELS || !w || !wd) return LGM_ERR_INVALID_ARGUMENT;
    const int n = cin * 9 * COUT;
    flip_weights<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>((const bf16*)w, (bf16*)wd, cin);
    return launch_check();
}

lgm_status lgm_cnn_gemm(const void* A, int32_t sam, int32_t sak, const void* Bm, int32_t sbk,
                        int32_t sbn, float* C, const float* bias, int32_t M, int32_t N, int32_t K,
                        int32_t relu, int32_t accumulate, void* stream) {
    if (!A || !Bm || !C || M < 1 || N < 1 || K < 1) return LGM_ERR_INVALID_ARGUMENT;
    const int warps = ((M + 15) / 16) * ((N + 7) / 8);
    gemm_small<<<(warps + 3) / 4, 128, 0, (cudaStream_t)stream>>>(
        (const bf16*)A, sam, sak, (const bf16*)Bm, sbk, sbn, C, bias, M, N, K, relu, accumulate);
    return launch_check();
}

lgm_status lgm_cnn_relu_pool_bwd(const void* act, const void* dP, void* dA, int32_t B, int32_t H,
                                 int32_t W, int32_t pooled, void* stream) {
    if (!act || !dP || !dA || B < 1 || H < 1 || W < 1) return LGM_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)B * H * W * COUT;
    relu_pool_bwd<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)act, (const bf16*)dP, (bf16*)dA, B, H, W, pooled);
    return launch_check();
}

lgm_status lgm_cnn_gap_fwd(const void* act, float* out32, void* out16, int32_t B, int32_t HW,
                           void* stream) {
    if (!act || !out32 || !out16 || B < 1 || HW < 1) return LGM_ERR_INVALID_ARGUMENT;
    gap_fwd<<<B, COUT, 0, (cudaStream_t)stream>>>((const bf16*)act, out32, (bf16*)out16, HW);
    return launch_check();
}

lgm_status lgm_cnn_gap_relu_bwd(const void* act, const float* dg, void* dA, int32_t B, int32_t HW,
                                void* stream) {
    if (!act || !dg || !dA || B < 1 || HW < 1) return LGM_ERR_INVALID_ARGUMENT;
    const size_t n = (size_t)B * HW * COUT;
    gap_relu_bwd<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const bf16*)act, dg, (bf16*)dA, B, HW);
    return launch_check();
}

lgm_status lgm_cnn_to_bf16(const float* in, void* out, int32_t n, const float* relu_mask,
                           void* stream) {
    if (!in || !out || n < 0) return LGM_ERR_INVALID_ARGUMENT;
    if (n == 0) return LGM_OK;
    f32_to_bf16<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(in, (bf16*)out, n,
                                                                    relu_mask != nullptr, relu_mask);
    return launch_check();
}

}  // extern "C"
