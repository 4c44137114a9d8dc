// lgm_api.cu -- C ABI of the Coulomb path: context, buffers, launches.
//
// Host side of the drop-in for OpenClHelper (src/langmuirCore/openclhelper.cpp):
// validation with status codes instead of qFatal, device buffers that stay
// resident, and the prep -> pair -> finalize launch sequence on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "langmuir_b200.h"
#include "lgm_context.hpp"
#include "lgm_cull.cuh"

using namespace lgm;

namespace {

thread_local std::string g_create_error;

constexpr int kMaxSplits = 64;
constexpr int kDrainIds = 35;       // Grid::m_specialAgentReserve (cubicgrid.cpp:22)

lgm_status fail(lgm_ctx* c, lgm_status st, const std::string& msg) {
    if (c) c->err = msg;
    return st;
}

lgm_status cuda_fail(lgm_ctx* c, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(c, LGM_ERR_CUDA, m);
}

#define LGM_CUDA(c, call)                                    \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail((c), e_, #call); \
    } while (0)

template <class T>
lgm_status grow_device(lgm_ctx* c, T** p, size_t* cap, size_t need) {
    if (need <= *cap && *p) return LGM_OK;
    size_t n = std::max(need, (size_t)(*cap * 3 / 2));
    n = std::max<size_t>(n, 256);
    if (*p) LGM_CUDA(c, cudaFree(*p));
    *p = nullptr;
    *cap = 0;
    LGM_CUDA(c, cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)));
    *cap = n;
    return LGM_OK;
}

template <class T>
lgm_status grow_host(lgm_ctx* c, T** p, size_t* cap, size_t need) {
    if (need <= *cap && *p) return LGM_OK;
    size_t n = std::max(need, (size_t)(*cap * 3 / 2));
    n = std::max<size_t>(n, 256);
    if (*p) LGM_CUDA(c, cudaFreeHost(*p));
    *p = nullptr;
    *cap = 0;
    LGM_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(p), n * sizeof(T)));
    *cap = n;
    return LGM_OK;
}

// ---- prep kernels ---------------------------------------------------------

// Source records (see lgm_pairs.cuh) in spatial order (prep_records).  The sources were
// counted into bins by lattice cell (bins_both) and scattered by bin
// (scatter_both, in no particular order inside a bin); slot j of that scatter
// takes its final place here: the bin's start plus its rank inside the bin by
// (site, index), so the order depends on the sources alone and the sums are
// deterministic.  bins_end[b] is the end of bin b after the scatter.  Entries
// n .. n_pad-1 are zero-charge padding at the origin; their weight is
// (q*m) * y = 0 * finite = 0.
__device__ __forceinline__ void source_record(int sj, int qj, int X, int XY, int Y, int volume,
                                              float4* __restrict__ geo, float2* __restrict__ qq,
                                              int dst, unsigned* err) {
    float a = 0.f, b = 0.f, cc = 0.f, d = -0.5f, qf = 0.f;
    if (sj < 0 || sj >= volume) {
        atomicOr(err, DEVERR_SOURCE_RANGE);
    } else {
        // Grid::getIndexX/Y/Z (cubicgrid.cpp:132-145), as kernel.cl:266-268.
        const int z = sj / XY, y = sj / X - z * Y, x = sj % X;
        a = -2.f * x; b = -2.f * y; cc = -2.f * z;
        d = (float)(x * x + y * y + z * z) - 0.5f;
        qf = (float)qj;
    }
    geo[2 * dst] = make_float4(a, a, b, b);
    geo[2 * dst + 1] = make_float4(cc, cc, d, d);
    qq[dst] = make_float2(qf, qf);
}

__device__ __forceinline__ void prep_source(const int j, const int32_t* __restrict__ s,
                                            const int32_t* __restrict__ q, int n, int n_pad,
                                            const int32_t* __restrict__ key,
                                            const int32_t* __restrict__ tmp,
                                            const int32_t* __restrict__ bins_end, int X, int Y,
                                            int XY, int volume, float4* __restrict__ geo,
                                            float2* __restrict__ qq, unsigned* err) {
    if (j >= n_pad) return;
    if (j >= n) {
        geo[2 * j] = make_float4(0.f, 0.f, 0.f, 0.f);
        geo[2 * j + 1] = make_float4(0.f, 0.f, -0.5f, -0.5f);
        qq[j] = make_float2(0.f, 0.f);
        return;
    }
    const int i = tmp[j];
    const int b = key[i];
    const int lo = b > 0 ? bins_end[b - 1] : 0, hi = bins_end[b];
    const int si = s[i];
    int rank = 0;
    for (int k = lo; k < hi; ++k) {
        const int o = tmp[k];
        const int so = s[o];
        rank += (so < si) | ((so == si) & (o < i));
    }
    source_record(si, q[i], X, XY, Y, volume, geo, qq, lo + rank, err);
}

// Physical targets: for each requested term the (possibly mirrored) target
// position.  Term order in `tgt`: direct, left image, right image (present
// ones only), each block t_pad long.  A left image is the direct sum at
// x' = -1 - x (distance x_i + x_j + 1, cubicgrid.cpp:117-120); a right image
// at x' = 2X - 1 - x.  all_sites != 0: target g is lattice site g (kernel 1).
__device__ __forceinline__ void prep_target(const int j, const int32_t* __restrict__ ts, int t,
                                            int t_pad, int all_sites, unsigned terms, int X,
                                            int Y, int XY, int volume, int shift,
                                            const int32_t* __restrict__ tkey,
                                            const int32_t* __restrict__ ttmp,
                                            const int32_t* __restrict__ bins_end,
                                            int32_t* __restrict__ perm, float4* __restrict__ tgt,
                                            unsigned* err) {
    if (j >= t_pad) return;  // j: the scatter slot
    // The target scattered to slot j goes to physical slot g: its bin's start
    // plus its rank inside the bin by index (perm[g] = target).  A target's
    // sum is split into the work items of its tile (the culled tiles), so its
    // tile, and with it the rounding of the item partials' sum, must not
    // depend on the scatter's order: with this rank the sums are a function
    // of the target list and the source set.  bins_end[b] is the end of bin b
    // after the scatter.
    // Every site (kernel 1): a cell's bin holds all its sites, and the rank
    // by index is the site's raster position inside the (edge-clipped) cell.
    int g = j, x = 0, y = 0, z = 0;
    if (j < t) {
        const int i = ttmp[j];
        const int b = tkey[i];
        const int lo = b > 0 ? bins_end[b - 1] : 0;
        const int sg = all_sites ? i : ts[i];
        if (sg < 0 || sg >= volume + kDrainIds) {
            atomicOr(err, DEVERR_TARGET_RANGE);
        } else {
            z = sg / XY; y = sg / X - z * Y; x = sg % X;
        }
        int rank = 0;
        if (all_sites) {
            const int c = 1 << shift;
            const int x0 = (x >> shift) << shift, y0 = (y >> shift) << shift;
            const int z0 = (z >> shift) << shift;
            const int cw = min(c, X - x0), ch = min(c, Y - y0);
            rank = ((z - z0) * ch + (y - y0)) * cw + (x - x0);
        } else {
            const int hi = bins_end[b];
            for (int k = lo; k < hi; ++k) rank += ttmp[k] < i;
        }
        g = lo + rank;
        perm[g] = i;
    }
    int slot = 0;
    for (int term = 0; term < 3; ++term) {
        if (!(terms & (1u << term))) continue;
        int xp = x;
        if (term == 1) xp = -1 - x;
        if (term == 2) xp = 2 * X - 1 - x;
        const float fx = (float)xp, fy = (float)y, fz = (float)z;
        // padding slots (g >= t) carry w = -1: the cull leaves them out of the
        // tiles' boxes, and their sums are never read
        tgt[(size_t)slot * t_pad + g] =
            make_float4(fx, fy, fz, g < t ? (float)(xp * xp + y * y + z * z) : -1.f);
        ++slot;
    }
}

// The target records (blocks [0, tb)) and the source records (the blocks
// after), one launch.
__global__ void prep_records(int tb, const int32_t* __restrict__ ts, int t, int t_pad,
                             int all_sites, unsigned terms, int X, int Y, int XY, int volume,
                             int shift, const int32_t* __restrict__ tkey,
                             const int32_t* __restrict__ ttmp,
                             const int32_t* __restrict__ tbins_end, int32_t* __restrict__ perm,
                             float4* __restrict__ tgt, const int32_t* __restrict__ s,
                             const int32_t* __restrict__ q, int n, int n_pad,
                             const int32_t* __restrict__ skey, const int32_t* __restrict__ stmp,
                             const int32_t* __restrict__ sbins_end, float4* __restrict__ geo,
                             float2* __restrict__ qq, unsigned* err) {
    pdl_wait();
    pdl_trigger();
    const int b = (int)blockIdx.x;
    if (b < tb)
        prep_target(b * (int)blockDim.x + (int)threadIdx.x, ts, t, t_pad, all_sites, terms, X, Y,
                    XY, volume, shift, tkey, ttmp, tbins_end, perm, tgt, err);
    else
        prep_source((b - tb) * (int)blockDim.x + (int)threadIdx.x, s, q, n, n_pad, skey, stmp,
                    sbins_end, X, Y, XY, volume, geo, qq, err);
}

// The last kernel of a call clears both bin arrays (their last reader,
// prep_records, has completed), so the next call's bins_both counts into
// zeros without a memset of its own.  Thread i of the grid (one row of the
// block) clears entries i, i + stride, ...
__device__ __forceinline__ void zero_bins(int32_t* __restrict__ bins, int nbins) {
    const int stride = (int)(gridDim.x * blockDim.x);
    for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < nbins; i += stride) bins[i] = 0;
}

// out[perm[g]] = prefactor * (sum over splits of the direct block - image
// blocks) of physical slot g.
__global__ void finalize(const double* __restrict__ part, int splits, int t_phys, int t,
                         int t_pad, int nterms, double prefactor,
                         const int32_t* __restrict__ perm, double* __restrict__ out,
                         int32_t* __restrict__ bins, int nbins, const unsigned* err,
                         unsigned* err_out) {
    pdl_wait();
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    zero_bins(bins, nbins);
    if (err_out && g == 0) *err_out = *err;
    if (g >= t) return;
    double total = 0.0;
    for (int slot = 0; slot < nterms; ++slot) {
        double s = 0.0;
        const double* p = part + (size_t)slot * t_pad + g;
        // eight loads in flight, then the adds in split order (same bits)
        int sp = 0;
        for (; sp + 8 <= splits; sp += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = p[(size_t)(sp + u) * t_phys];
#pragma unroll
            for (int u = 0; u < 8; ++u) s += v[u];
        }
        for (; sp < splits; ++sp) s += p[(size_t)sp * t_phys];
        total = (slot == 0) ? s : total - s;
    }
    out[perm[g]] = prefactor * total;
}

// Counting sort of the targets and of the sources by lattice cell (the
// spatial order the SKIP and culled pair tiles run in).  bins_both: the bin of
// every target and every source -- the Morton rank of its cell, sites beyond
// the lattice (drains, or ids the prep flags as out of range) in the last bin
// -- and the bin counts (target bins tbins, source bins sbins).
__device__ __forceinline__ int cell_bin(int sg, int X, int Y, int XY, int volume, int shift,
                                        int cells_x, int cells_y,
                                        const int32_t* __restrict__ cell_rank, int ncells) {
    if (sg < 0 || sg >= volume) return ncells;
    const int z = sg / XY, y = sg / X - z * Y, x = sg % X;
    return cell_rank[(x >> shift) + cells_x * ((y >> shift) + cells_y * (z >> shift))];
}

__global__ void bins_both(const int32_t* __restrict__ ts, int t, int all_sites,
                          const int32_t* __restrict__ ss, int n, int X, int Y, int XY, int volume,
                          int shift, int cells_x, int cells_y,
                          const int32_t* __restrict__ cell_rank, int ncells,
                          int32_t* __restrict__ tkey, int32_t* __restrict__ tbins,
                          int32_t* __restrict__ skey, int32_t* __restrict__ sbins,
                          int32_t* __restrict__ done) {
    __shared__ int s_last;
    pdl_wait();
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < t) {
        const int b = cell_bin(all_sites ? g : ts[g], X, Y, XY, volume, shift, cells_x, cells_y,
                               cell_rank, ncells);
        tkey[g] = b;
        atomicAdd(&tbins[b], 1);
    }
    if (g < n) {
        const int b =
            cell_bin(ss[g], X, Y, XY, volume, shift, cells_x, cells_y, cell_rank, ncells);
        skey[g] = b;
        atomicAdd(&sbins[b], 1);
    }
    // The last block to finish turns both counts into exclusive scans in
    // place (the counts were added by atomics in L2; this block read none of
    // them before, and fences after seeing the others done).
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    block_exclusive_scan(tbins, ncells + 1);
    block_exclusive_scan(sbins, ncells + 1);
    if (threadIdx.x == 0) *done = 0;  // every block has counted itself: ready for the next call
}


// ttmp[slot] = target and stmp[slot] = source: each takes the next slot of
// its bin, in no particular order inside the bin; prep_target and
// prep_source (prep_records) fix the final order.
__global__ void scatter_both(const int32_t* __restrict__ tkey, int t, int32_t* __restrict__ tbins,
                             int32_t* __restrict__ ttmp, const int32_t* __restrict__ skey, int n,
                             int32_t* __restrict__ sbins, int32_t* __restrict__ stmp) {
    pdl_wait();
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < t) ttmp[atomicAdd(&tbins[tkey[g]], 1)] = g;
    if (g < n) stmp[atomicAdd(&sbins[skey[g]], 1)] = g;
}

// out[perm[g]] = prefactor * (sum of the item partials of the direct slot -
// those of the image slots) of target g, for the culled pair sums.  A block
// of 32 x 3 threads takes 32 targets: warp y sums term slot y's partials of
// each target in item order, sixteen items in flight; warp 0 then combines the
// slots through shared memory.
__global__ void __launch_bounds__(96) finalize_items(const double* __restrict__ part,
                                                     const int* __restrict__ tile_first,
                                                     const int* __restrict__ tile_items,
                                                     int tile_size, int t, int t_pad, int nterms,
                                                     double prefactor,
                                                     const int32_t* __restrict__ perm,
                                                     double* __restrict__ out,
                                                     int32_t* __restrict__ bins, int nbins,
                                                     const unsigned* err, unsigned* err_out) {
    constexpr int kRows = 16;  // loads in flight (a tile has at most 32 items)
    __shared__ double s_sum[3][32];
    pdl_wait();
    pdl_trigger();
    const int g = blockIdx.x * 32 + (int)threadIdx.x, slot = (int)threadIdx.y;
    const int dst = slot == 0 && g < t ? perm[g] : 0;  // loaded ahead of the sums
    if (slot == 0) zero_bins(bins, nbins);
    if (err_out && g == 0 && slot == 0) *err_out = *err;
    double sum = 0.0;
    if (g < t && slot < nterms) {
        const int p = slot * t_pad + g;
        const int tile = p / tile_size, loc = p - tile * tile_size;
        const int n = tile_items[tile];
        const double* q = part + (size_t)tile_first[tile] * tile_size + loc;
        for (int i = 0; i < n; i += kRows) {
            double v[kRows];
#pragma unroll
            for (int u = 0; u < kRows; ++u)
                v[u] = i + u < n ? q[(size_t)(i + u) * tile_size] : 0.0;
#pragma unroll
            for (int u = 0; u < kRows; ++u)
                if (i + u < n) sum += v[u];
        }
    }
    s_sum[slot][threadIdx.x] = sum;
    __syncthreads();
    if (slot == 0 && g < t) {
        const int x = (int)threadIdx.x;
        out[dst] = prefactor * (s_sum[0][x] - s_sum[1][x] - s_sum[2][x]);
    }
}

__global__ void fill_zero(double* out, int t, const unsigned* err, unsigned* err_out) {
    pdl_wait();
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (err_out && g == 0) *err_out = *err;
    if (g < t) out[g] = 0.0;
}

// FP64 path: every term in double, 1/sqrt and erf of the CUDA runtime.
// Sources staged in shared memory by plain loads; one thread per physical
// target and split.
constexpr int kF64Threads = 256;
constexpr int kF64Tile = 512;

__global__ void __launch_bounds__(kF64Threads)
pair_kernel_f64(const float4* __restrict__ geo, const float2* __restrict__ qq, int n_pad,
                int splits, const float4* __restrict__ tgt, int t_phys, double* __restrict__ part,
                int c2, int kind, double erffactor) {
    __shared__ int4 s_g[kF64Tile];  // x, y, z, q
    pdl_wait();
    pdl_trigger();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int split = blockIdx.y;
    const int j_begin = (int)((long long)split * n_pad / splits);
    const int j_end = (int)((long long)(split + 1) * n_pad / splits);
    float4 tp = p < t_phys ? tgt[p] : make_float4(0.f, 0.f, 0.f, 0.f);
    // target coordinates are exact small integers
    const int tx = (int)tp.x, ty = (int)tp.y, tz = (int)tp.z;
    double acc = 0.0;
    for (int j0 = j_begin; j0 < j_end; j0 += kF64Tile) {
        const int m = min(kF64Tile, j_end - j0);
        __syncthreads();
        for (int k = threadIdx.x; k < m; k += blockDim.x) {
            const float4 g0 = geo[2 * (j0 + k)], g1 = geo[2 * (j0 + k) + 1];
            s_g[k] = make_int4((int)(-0.5f * g0.x), (int)(-0.5f * g0.z), (int)(-0.5f * g1.x),
                               (int)qq[j0 + k].x);
        }
        __syncthreads();
        for (int k = 0; k < m; ++k) {
            const int4 sk = s_g[k];
            const int dx = tx - sk.x, dy = ty - sk.y, dz = tz - sk.z;
            const int r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0 && r2 < c2) {
                const double r = (double)r2;
                if (kind == 0) {
                    acc += (double)sk.w * (1.0 / sqrt(r));
                } else {
                    const double rr = sqrt(r);
                    acc += (double)sk.w * erf(erffactor * rr) / rr;
                }
            }
        }
    }
    if (p < t_phys) part[(size_t)split * t_phys + p] = acc;
}

// ---- launch plumbing --------------------------------------------------------

// Launches a kernel of a call's chain.  With overlap on it carries the
// programmatic stream serialization attribute: the kernel may be scheduled
// while the one ahead of it in the stream is still running, and waits for it
// in pdl_wait() (lgm_device.cuh) before touching memory, so the launch
// latency between the chain's kernels overlaps the kernel ahead.
template <typename... P, typename... A>
cudaError_t launch_chain(bool overlap, void (*k)(P...), dim3 grid, dim3 block, size_t smem,
                         cudaStream_t st, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, static_cast<P>(args)...);
}

using PairFn = void (*)(PairArgs);
using CulledFn = void (*)(PairArgs, CullArgs);

// Compiled tile variants of the pair kernel: threads per CTA, target pairs per
// thread, FP32 run length.  fn[0] point/rsqrt, fn[1] gauss/rsqrt, fn[2] table.
// skip: warp-owned spatially sorted targets with the per-source warp vote
// (the rsqrt paths; the table path runs the plain tile).  cull: the work-list
// kernel of lgm_cull.cuh over the live source chunks of each tile, per_item
// chunks per work item (cfn[] instead of fn[]).
struct Variant {
    int nt, rp, sub, skip, cull, per_item;
    PairFn fn[4];
    CulledFn cfn[4];  // [3]: the FP64-table path (culled variants only)
    int ws = 0;       // warp-specialised culled kernel: its stages (0: not)
};
#define LGM_VARIANT_S(NT, RP, SUB, SK)                                                    \
    Variant {                                                                             \
        NT, RP, SUB, SK, 0, 0,                                                            \
            {&pair_kernel<0, 0, NT, RP, SUB, false, SK>,                                  \
             &pair_kernel<1, 0, NT, RP, SUB, false, SK>, &pair_kernel<0, 1, NT, RP, SUB>,  \
             nullptr},                                                                    \
        {                                                                                 \
            nullptr, nullptr, nullptr, nullptr                                            \
        }                                                                                 \
    }
#define LGM_VARIANT(NT, RP, SUB) LGM_VARIANT_S(NT, RP, SUB, false)
#define LGM_VARIANT_SKIP(NT, RP, SUB) LGM_VARIANT_S(NT, RP, SUB, true)
#define LGM_VARIANT_CULL(NT, RP, SUB, K)                                                      \
    Variant {                                                                                 \
        NT, RP, SUB, 1, 1, K, {nullptr, nullptr, nullptr, nullptr}, {                         \
            &pair_kernel_culled<0, 0, NT, RP, SUB>, &pair_kernel_culled<1, 0, NT, RP, SUB>,   \
                &pair_kernel_culled<0, 1, NT, RP, SUB>, &pair_kernel_culled<0, 2, NT, RP, SUB> \
        }                                                                                     \
    }
#define LGM_VARIANT_CULL_WS(NW, RP, SUB, K, S, MINB, PIPE)                                  \
    Variant {                                                                                 \
        NW * 32, RP, SUB, 1, 1, K, {nullptr, nullptr, nullptr, nullptr},                      \
            {&pair_kernel_culled_ws<0, 0, NW, RP, SUB, S, MINB, false, PIPE>,                 \
             &pair_kernel_culled_ws<1, 0, NW, RP, SUB, S, MINB, false, PIPE>,                 \
             &pair_kernel_culled_ws<0, 1, NW, RP, SUB, S, MINB>,                              \
             &pair_kernel_culled_ws<0, 2, NW, RP, SUB, S, MINB>},                             \
            S                                                                                 \
    }
// VOTE: sources per warp vote of the MUFU path (0: none; lgm_cull.cuh)
#define LGM_VARIANT_CULL_WSV(NW, RP, SUB, K, S, MINB, VOTE)                                  \
    Variant {                                                                                 \
        NW * 32, RP, SUB, 1, 1, K, {nullptr, nullptr, nullptr, nullptr},                      \
            {&pair_kernel_culled_ws<0, 0, NW, RP, SUB, S, MINB, false, false, VOTE>,          \
             &pair_kernel_culled_ws<1, 0, NW, RP, SUB, S, MINB, false, false, VOTE>,          \
             &pair_kernel_culled_ws<0, 1, NW, RP, SUB, S, MINB>,                              \
             &pair_kernel_culled_ws<0, 2, NW, RP, SUB, S, MINB>},                             \
            S                                                                                 \
    }
const Variant kVariants[] = {
    LGM_VARIANT(128, 4, 16),       LGM_VARIANT(128, 4, 8),        LGM_VARIANT(128, 2, 16),
    LGM_VARIANT(128, 8, 16),       LGM_VARIANT(256, 4, 16),       LGM_VARIANT(64, 4, 16),
    LGM_VARIANT(128, 4, 32),       LGM_VARIANT(256, 2, 16),       LGM_VARIANT_SKIP(128, 4, 32),
    LGM_VARIANT_SKIP(128, 4, 16),  LGM_VARIANT_SKIP(128, 2, 32),  LGM_VARIANT_SKIP(64, 4, 32),
    LGM_VARIANT_SKIP(64, 3, 32),   LGM_VARIANT_SKIP(128, 3, 32),
    LGM_VARIANT_CULL(128, 4, 16, 2), LGM_VARIANT_CULL(128, 4, 16, 1),
    LGM_VARIANT_CULL(128, 4, 16, 4), LGM_VARIANT_CULL(128, 2, 16, 2),
    LGM_VARIANT_CULL(64, 4, 16, 2),  LGM_VARIANT_CULL(128, 4, 8, 2),
    LGM_VARIANT_CULL(64, 2, 16, 2),
    // warp-specialised: (target warps, target pairs, run, chunks per item,
    // stages, CTAs per SM); the register bound counts the producer warp
    LGM_VARIANT_CULL_WS(4, 4, 16, 2, 4, 4, false), LGM_VARIANT_CULL_WS(8, 2, 16, 2, 4, 3, false),
    LGM_VARIANT_CULL_WS(4, 2, 16, 2, 4, 5, false), LGM_VARIANT_CULL_WS(7, 2, 16, 2, 4, 3, false),
    LGM_VARIANT_CULL_WS(4, 4, 16, 4, 4, 4, false),
    // 4 CTAs of 4 target warps and 2 target pairs per thread measured best on
    // the 256x256x16 and 128x128x64 workloads (96 registers; the 5-CTA bound
    // of 72 registers was 36% slower); the next source's r^2 ahead of each
    // vote (PIPE) measured the same
    LGM_VARIANT_CULL_WS(4, 2, 16, 2, 4, 4, true), LGM_VARIANT_CULL_WS(4, 2, 16, 2, 4, 4, false),
    LGM_VARIANT_CULL_WS(2, 2, 16, 2, 4, 6, true), LGM_VARIANT_CULL_WS(4, 2, 16, 3, 4, 4, false),
    LGM_VARIANT_CULL_WS(4, 2, 16, 1, 4, 4, true), LGM_VARIANT_CULL_WS(4, 2, 16, 4, 4, 4, false),
    // one vote per 2 or 4 sources, or none
    LGM_VARIANT_CULL_WSV(4, 2, 16, 2, 4, 4, 2), LGM_VARIANT_CULL_WSV(4, 2, 16, 2, 4, 4, 0),
    LGM_VARIANT_CULL_WSV(4, 2, 16, 2, 4, 4, 4),
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));
static_assert(kNumVariants <= (int)(sizeof(lgm_ctx::bps) / sizeof(lgm_ctx::bps[0])),
              "lgm_ctx::bps holds every variant");
// warp-specialised culled, 4 target warps, 2 target pairs, runs of 16, 2
// chunks per item, one vote per 2 sources (2% faster than a vote per source
// on the 256x256x16 and 128x128x64 workloads, the same bits)
constexpr int kDefaultVariant = 32;

const void* kernel_of(const Variant& V, int fi) {
    return V.cull ? reinterpret_cast<const void*>(V.cfn[fi])
                  : reinterpret_cast<const void*>(V.fn[fi]);
}

// Threads of a CTA (a warp-specialised variant adds its producer warp) and
// dynamic shared memory for path index fi with table entries 0 .. tab_k.
int variant_threads(const Variant& V) { return V.nt + (V.ws ? 32 : 0); }
size_t variant_smem(const Variant& V, int fi, int tab_k) {
    if (V.ws) return ws_smem_bytes(V.ws, tab_k, fi == 3 ? 8 : 4);
    return fi == 3 ? pair_smem_bytes64(tab_k) : pair_smem_bytes(tab_k);
}

int fn_index(int kind, int path) {
    if (path == LGM_PATH_TABLE64) return 3;  // one kernel: the table holds w for the kind
    if (path == LGM_PATH_TABLE) return 2;
    return kind == LGM_GAUSS ? 1 : 0;
}

// Size bucket of a pair launch: half-octaves of physical targets and chunks.
uint64_t tune_key(int kind, int path, int t_phys, int n_chunks) {
    auto hb = [](int x) { return (uint64_t)std::lround(2.0 * std::log2((double)std::max(x, 1))); };
    return ((uint64_t)kind << 60) | ((uint64_t)path << 56) | (hb(t_phys) << 28) | hb(n_chunks);
}

int popcount3(unsigned terms) {
    return ((terms & 1u) ? 1 : 0) + ((terms & 2u) ? 1 : 0) + ((terms & 4u) ? 1 : 0);
}

// Source and target records for a call (see lgm_pairs.cuh).
struct Shape {
    int nterms, n_pad, n_chunks, t_pad, t_phys;
};

Shape shape_of(int n, int t, unsigned terms) {
    Shape sh;
    sh.nterms = popcount3(terms);
    sh.n_pad = (n + CH - 1) / CH * CH;
    sh.n_chunks = sh.n_pad / CH;
    sh.t_pad = (t + 63) / 64 * 64;
    sh.t_phys = sh.nterms * sh.t_pad;
    return sh;
}

lgm_status prep(lgm_ctx* c, unsigned terms, const int32_t* d_src, const int32_t* d_q, int n,
                const int32_t* d_tgt_site, int t, int all_sites, const Shape& sh,
                cudaStream_t st) {
    const lgm_config& cf = c->cfg;
    lgm_status s;
    if ((s = grow_device(c, &c->d_geo, &c->geo_cap, (size_t)sh.n_pad * 2)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_qq, &c->qq_cap, (size_t)sh.n_pad)) != LGM_OK) return s;
    // room for the widest target tile of any variant
    if ((s = grow_device(c, &c->d_tgt, &c->tgt_cap, (size_t)sh.t_phys + 4096)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_key, &c->key_cap, (size_t)t)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_perm, &c->perm_cap, (size_t)t)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_ttmp, &c->ttmp_cap, (size_t)t)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_skey, &c->skey_cap, (size_t)n)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_stmp, &c->stmp_cap, (size_t)n)) != LGM_OK) return s;
    // targets and sources in spatial order: bins, scans, scatters.  Both bin
    // arrays and the bins_both block counter behind them start at zero: the
    // last kernel of the previous call cleared them (bins_both's last block
    // clears the counter), else one memset does.
    if (!c->bins_clean)
        LGM_CUDA(c, cudaMemsetAsync(c->d_bins, 0, sizeof(int32_t) * (2 * c->bins_stride + 4), st));
    c->bins_clean = false;
    const bool ov = c->overlap;
    const int tb = (std::max(t, n) + 255) / 256;
    LGM_CUDA(c, launch_chain(ov, bins_both, tb, 256, 0, st, d_tgt_site, t, all_sites, d_src, n,
                             cf.grid_x, cf.grid_y, c->xy, c->volume, c->cell_shift, c->cells_x,
                             c->cells_y, c->d_cell_rank, c->ncells, c->d_key, c->d_bins,
                             c->d_skey, c->d_sbins, c->d_bins + 2 * c->bins_stride));
    LGM_CUDA(c, launch_chain(ov, scatter_both, tb, 256, 0, st, c->d_key, t, c->d_bins, c->d_ttmp,
                             c->d_skey, n, c->d_sbins, c->d_stmp));
    const int ptb = (sh.t_pad + 255) / 256, psb = (sh.n_pad + 255) / 256;
    LGM_CUDA(c, launch_chain(ov, prep_records, ptb + psb, 256, 0, st, ptb, d_tgt_site, t, sh.t_pad,
                             all_sites, terms, cf.grid_x, cf.grid_y, c->xy, c->volume,
                             c->cell_shift, c->d_key, c->d_ttmp, c->d_bins, c->d_perm, c->d_tgt,
                             d_src, d_q, n, sh.n_pad, c->d_skey, c->d_stmp, c->d_sbins, c->d_geo,
                             c->d_qq, c->d_err));
    return LGM_OK;
}

// Splits of the source range for variant v: as many as fill kSplitWaves
// waves of resident CTAs, never more than the chunks.  With the warp skip the
// CTAs of one launch do uneven work (tiles near few charges, image tiles far
// from the electrode skip most sources), and three waves of smaller CTAs let
// the block scheduler even it out; more waves cost more in the FP64 partials
// that finalize sums than they save (256x256x16 lattice, 20,970 charges,
// images at both electrodes: 1 wave 0.647 ms, 3 waves 0.607 ms, 8 waves
// 0.614 ms per call).
constexpr int kSplitWaves = 3;
int splits_for(const lgm_ctx* c, int v, int fi, const Shape& sh, int* tiles_out) {
    const Variant& V = kVariants[v];
    const int tiles = (sh.t_phys + V.nt * 2 * V.rp - 1) / (V.nt * 2 * V.rp);
    const int capacity = c->sm_count * std::max(1, c->bps[v][fi]);
    *tiles_out = tiles;
    return std::max(1, std::min({kMaxSplits, kSplitWaves * capacity / tiles, sh.n_chunks}));
}

// Culled variant v: chunk boxes, the cull, the persistent pair kernel (one
// wave of resident CTAs).  *splits_out = 0 tells the caller to finalize from
// the item partials.
lgm_status launch_culled(lgm_ctx* c, int kind, int v, const Shape& sh, const PairArgs& A,
                         cudaStream_t st, int* splits_out) {
    const Variant& V = kVariants[v];
    const int fi = fn_index(kind, c->cfg.path);
    const int TS = V.nt * 2 * V.rp;
    const int tiles = (sh.t_phys + TS - 1) / TS;
    const int max_items = std::min(kMaxItemsPerTile, (sh.n_chunks + V.per_item - 1) / V.per_item);
    if (V.nt / 32 > kMaxSegments) return fail(c, LGM_ERR_STATE, "culled variant wider than the cull");
    const size_t item_cap = (size_t)tiles * std::max(1, max_items);
    lgm_status s;
    if ((s = grow_device(c, &c->d_cbox, &c->cbox_cap, (size_t)sh.n_chunks)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_gbox, &c->gbox_cap, (size_t)sh.n_chunks * kGroupsPerChunk)) !=
        LGM_OK)
        return s;
    if ((s = grow_device(c, &c->d_live, &c->live_cap, (size_t)tiles * sh.n_chunks)) != LGM_OK)
        return s;
    if ((s = grow_device(c, &c->d_items, &c->items_cap, item_cap)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_tile_first, &c->tfirst_cap, (size_t)tiles)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_tile_items, &c->titems_cap, (size_t)tiles)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_part, &c->part_cap, item_cap * TS)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_order, &c->order_cap, item_cap)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_oitems, &c->oitems_cap, item_cap)) != LGM_OK) return s;
    PairArgs P = A;
    P.part = c->d_part;
    CullArgs C;
    C.n_chunks = sh.n_chunks;
    C.cbox = reinterpret_cast<Box*>(c->d_cbox);
    C.gbox = reinterpret_cast<Box*>(c->d_gbox);
    C.tgt = c->d_tgt;
    C.t_phys = sh.t_phys;
    C.c2 = c->cfg.electrostatic_cutoff * c->cfg.electrostatic_cutoff;
    C.tile_size = TS;
    C.per_item = V.per_item;
    C.max_items = std::max(1, max_items);
    C.live = c->d_live;
    C.live_stride = sh.n_chunks;
    C.items = c->d_items;
    C.item_count = c->d_item_count;
    C.work = c->d_item_count + 1;
    C.tile_first = c->d_tile_first;
    C.tile_items = c->d_tile_items;
    // the items largest first (costs from the pair kernel's warp segments)
    C.warp_targets = 64 * V.rp;
    C.hist = c->d_cost_hist;
    C.order = c->d_order;
    C.oitems = c->d_oitems;
    C.done = c->d_item_count + 2;
    if (c->counting) {
        LGM_CUDA(c, cudaMemsetAsync(c->d_examined, 0, sizeof(unsigned long long), st));
        C.examined = c->d_examined;
        c->count_pending = true;
    }
    const bool ov = c->overlap;
    LGM_CUDA(c, launch_chain(ov, chunk_boxes_kernel, sh.n_chunks, CH, 0, st, P, C));
    // its last block orders the items
    LGM_CUDA(c, launch_chain(ov, cull_kernel, tiles, kCullThreads, 0, st, C));
    // timing on: the events bracket the pair kernel alone (recorded again here)
    if (c->timing) LGM_CUDA(c, cudaEventRecord(c->ev_pair0, st));
    const int grid = c->sm_count * std::max(1, c->bps[v][fi]);
    LGM_CUDA(c, launch_chain(ov, V.cfn[fi], grid, variant_threads(V),
                             variant_smem(V, fi, P.tab_k), st, P, C));
    c->last.ctas = grid;
    c->last.threads = variant_threads(V);
    c->last.targets_per_thread = 2 * V.rp;
    c->last.variant = v;
    c->last.splits = 0;
    *splits_out = 0;
    return LGM_OK;
}

lgm_status launch_pair(lgm_ctx* c, int kind, int v, const Shape& sh, cudaStream_t st,
                       int* splits_out) {
    const lgm_config& cf = c->cfg;
    const int fi = fn_index(kind, cf.path);
    if (kVariants[v].cull) {
        PairArgs A;
        A.geo = c->d_geo; A.qq = c->d_qq; A.n_chunks = sh.n_chunks; A.splits = 1;
        A.tgt = c->d_tgt; A.t_phys = sh.t_phys;
        A.c2 = (float)(cf.electrostatic_cutoff * cf.electrostatic_cutoff);
        A.err = c->d_err;
        if (cf.path == LGM_PATH_TABLE64) {
            A.tab64 = kind == LGM_GAUSS ? c->d_gtab64 : c->d_rtab64;
            A.tab_k = c->rtab_k;  // both hold every r^2 <= c^2 (entries 0 and c^2 are 0)
        } else if (cf.path == LGM_PATH_TABLE) {
            A.tab = kind == LGM_GAUSS ? c->d_gtab : c->d_rtab;
            A.tab_k = kind == LGM_GAUSS ? c->gtab_k : c->rtab_k;
        } else {
            A.tab = c->d_gtab;
            A.tab_k = kind == LGM_GAUSS ? c->gtab_k : 0;
        }
        return launch_culled(c, kind, v, sh, A, st, splits_out);
    }
    int tiles;
    const int splits = splits_for(c, v, fi, sh, &tiles);
    lgm_status s;
    if ((s = grow_device(c, &c->d_part, &c->part_cap, (size_t)splits * sh.t_phys)) != LGM_OK)
        return s;
    PairArgs A;
    A.geo = c->d_geo; A.qq = c->d_qq; A.n_chunks = sh.n_chunks; A.splits = splits;
    A.tgt = c->d_tgt; A.t_phys = sh.t_phys; A.part = c->d_part;
    A.c2 = (float)(cf.electrostatic_cutoff * cf.electrostatic_cutoff);
    A.err = c->d_err;
    if (cf.path == LGM_PATH_TABLE) {
        A.tab = kind == LGM_GAUSS ? c->d_gtab : c->d_rtab;  // both hold every r^2 < c^2
        A.tab_k = kind == LGM_GAUSS ? c->gtab_k : c->rtab_k;
    } else {
        A.tab = c->d_gtab;
        A.tab_k = kind == LGM_GAUSS ? c->gtab_k : 0;
    }
    const Variant& V = kVariants[v];
    dim3 grid(tiles, splits);
    LGM_CUDA(c, launch_chain(c->overlap, V.fn[fi], grid, V.nt, pair_smem_bytes(A.tab_k), st, A));
    c->last.ctas = grid.x * grid.y;
    c->last.threads = V.nt;
    c->last.targets_per_thread = 2 * V.rp;
    c->last.variant = v;
    *splits_out = splits;
    return LGM_OK;
}

int choose_variant(const lgm_ctx* c, int kind, const Shape& sh) {
    int v = kDefaultVariant;
    if (c->forced_variant >= 0) {
        v = c->forced_variant;
    } else {
        auto it = c->tune_cache.find(tune_key(kind, c->cfg.path, sh.t_phys, sh.n_chunks));
        if (it != c->tune_cache.end()) v = it->second;
    }
    // the FP64-table path is served by the culled variants only
    if (c->cfg.path == LGM_PATH_TABLE64 && !kVariants[v].cull) v = kDefaultVariant;
    return v;
}

// Shared launch sequence.  d_src/d_q: n sources; d_tgt_site: t targets (or
// all lattice sites when all_sites).  Everything on `st`.
lgm_status launch_potentials(lgm_ctx* c, int kind, unsigned terms, const int32_t* d_src,
                             const int32_t* d_q, int n, const int32_t* d_tgt_site, int t,
                             int all_sites, double* d_out, cudaStream_t st,
                             unsigned* err_out = nullptr) {
    const lgm_config& cf = c->cfg;
    c->last = lgm_launch_info{};
    c->last.pair_kernel_ms = -1.f;
    c->last.variant = -1;
    c->last.pairs_examined = -1;
    c->timed_pending = false;
    c->count_pending = false;
    if (t == 0) return LGM_OK;
    if (n == 0) {
        LGM_CUDA(c, launch_chain(c->overlap, fill_zero, (t + 255) / 256, 256, 0, st, d_out, t,
                                 c->d_err, err_out));
        c->last.kernel_launches = 1;
        return LGM_OK;
    }
    const Shape sh = shape_of(n, t, terms);
    lgm_status s;
    if ((s = prep(c, terms, d_src, d_q, n, d_tgt_site, t, all_sites, sh, st)) != LGM_OK) return s;
    int splits = 1;
    if (c->timing) LGM_CUDA(c, cudaEventRecord(c->ev_pair0, st));
    if (cf.precision == LGM_PREC_FP64) {
        const double erffactor =
            cf.coulomb_gaussian_sigma > 0 ? 1.0 / (std::sqrt(2.0) * cf.coulomb_gaussian_sigma) : 0.0;
        const int ctas = (sh.t_phys + kF64Threads - 1) / kF64Threads;
        splits = std::max(1, std::min({kMaxSplits, (c->sm_count * 8) / std::max(1, ctas),
                                       (sh.n_pad + kF64Tile - 1) / kF64Tile}));
        if ((s = grow_device(c, &c->d_part, &c->part_cap, (size_t)splits * sh.t_phys)) != LGM_OK)
            return s;
        dim3 grid(ctas, splits);
        LGM_CUDA(c, launch_chain(c->overlap, pair_kernel_f64, grid, kF64Threads, 0, st, c->d_geo,
                                 c->d_qq, sh.n_pad, splits, c->d_tgt, sh.t_phys, c->d_part,
                                 cf.electrostatic_cutoff * cf.electrostatic_cutoff, kind,
                                 erffactor));
        c->last.ctas = grid.x * grid.y;
        c->last.threads = kF64Threads;
        c->last.targets_per_thread = 1;
    } else {
        if ((s = launch_pair(c, kind, choose_variant(c, kind, sh), sh, st, &splits)) != LGM_OK)
            return s;
    }
    if (c->timing) {
        LGM_CUDA(c, cudaEventRecord(c->ev_pair1, st));
        c->timed_pending = true;
    }
    // the last kernel also clears both bin arrays for the next call
    const int nbins = 2 * c->bins_stride;
    if (splits > 0) {
        LGM_CUDA(c, launch_chain(c->overlap, finalize, (t + 255) / 256, 256, 0, st, c->d_part,
                                 splits, sh.t_phys, t, sh.t_pad, sh.nterms,
                                 cf.electrostatic_prefactor, c->d_perm, d_out, c->d_bins, nbins,
                                 c->d_err, err_out));
        c->last.kernel_launches = 5;  // bins (+ scan), scatter, records, pair, finalize
    } else {
        const Variant& V = kVariants[c->last.variant];
        LGM_CUDA(c, launch_chain(c->overlap, finalize_items, (t + 31) / 32, dim3(32, 3), 0, st,
                                 c->d_part, c->d_tile_first, c->d_tile_items, V.nt * 2 * V.rp, t,
                                 sh.t_pad, sh.nterms, cf.electrostatic_prefactor, c->d_perm, d_out,
                                 c->d_bins, nbins, c->d_err, err_out));
        c->last.kernel_launches = 7;  // bins (+ scan), scatter, records, boxes, cull, pair, finalize
    }
    c->bins_clean = true;
    c->last.pairs_tested = (int64_t)sh.nterms * t * (int64_t)n;
    c->last.splits = splits;
    return LGM_OK;
}

// The status of device error word e (read back into c->h_err); a nonzero word
// is cleared on the device for the next call.
lgm_status device_error_status(lgm_ctx* c, cudaStream_t st, unsigned e) {
    if (e == 0) return LGM_OK;
    LGM_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), st));
    LGM_CUDA(c, cudaStreamSynchronize(st));
    if (e & DEVERR_TIMEOUT) return fail(c, LGM_ERR_TIMEOUT, "a bounded device wait ran out");
    if (e & DEVERR_SOURCE_RANGE)
        return fail(c, LGM_ERR_OUT_OF_RANGE, "a source site lies outside [0, volume)");
    if (e & DEVERR_TARGET_RANGE)
        return fail(c, LGM_ERR_OUT_OF_RANGE, "a target site lies outside [0, volume + 35)");
    return fail(c, LGM_ERR_STATE, "device reported an inconsistent state");
}

lgm_status check_device_error(lgm_ctx* c, cudaStream_t st) {
    LGM_CUDA(c, cudaMemcpyAsync(c->h_err, c->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    LGM_CUDA(c, cudaStreamSynchronize(st));
    return device_error_status(c, st, *c->h_err);
}

lgm_status check_common(lgm_ctx* c, int kind, unsigned terms, int n, int t) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    c->err.clear();
    if (kind != LGM_POINT && kind != LGM_GAUSS)
        return fail(c, LGM_ERR_INVALID_ARGUMENT, "kind must be LGM_POINT or LGM_GAUSS");
    if (kind == LGM_GAUSS && !(c->cfg.coulomb_gaussian_sigma > 0))
        return fail(c, LGM_ERR_INVALID_ARGUMENT, "LGM_GAUSS needs coulomb.gaussian.sigma > 0");
    if (terms == 0 || (terms & ~7u) || !(terms & LGM_TERM_DIRECT))
        return fail(c, LGM_ERR_INVALID_ARGUMENT,
                    "terms must include LGM_TERM_DIRECT and only the three term bits");
    if (n < 0 || t < 0) return fail(c, LGM_ERR_INVALID_ARGUMENT, "negative size");
    if (c->cfg.max_charges > 0 && n > c->cfg.max_charges)
        return fail(c, LGM_ERR_CAPACITY, "more sources than max_charges");
    if (c->cfg.max_targets > 0 && t > c->cfg.max_targets)
        return fail(c, LGM_ERR_CAPACITY, "more targets than max_targets");
    return LGM_OK;
}


lgm_status check_sites(lgm_ctx* c, const int32_t* src, int n, const int32_t* tgt, int t) {
    for (int j = 0; j < n; ++j)
        if (src[j] < 0 || src[j] >= c->volume) {
            char b[128];
            std::snprintf(b, sizeof b, "source %d: site %d outside [0, %d)", j, src[j], c->volume);
            return fail(c, LGM_ERR_OUT_OF_RANGE, b);
        }
    for (int g = 0; g < t; ++g)
        if (tgt[g] < 0 || tgt[g] >= c->volume + kDrainIds) {
            char b[128];
            std::snprintf(b, sizeof b, "target %d: site %d outside [0, %d)", g, tgt[g],
                          c->volume + kDrainIds);
            return fail(c, LGM_ERR_OUT_OF_RANGE, b);
        }
    return LGM_OK;
}

}  // namespace

// ---- ABI ----------------------------------------------------------------------

extern "C" {

int32_t lgm_abi_version(void) { return LGM_ABI_VERSION; }

const char* lgm_status_string(lgm_status s) {
    switch (s) {
    case LGM_OK: return "ok";
    case LGM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LGM_ERR_OUT_OF_RANGE: return "site out of range";
    case LGM_ERR_CUDA: return "CUDA error";
    case LGM_ERR_NO_DEVICE: return "no usable sm_100 device";
    case LGM_ERR_CAPACITY: return "capacity exceeded";
    case LGM_ERR_TIMEOUT: return "device wait timed out";
    case LGM_ERR_PARSE: return "parse error";
    case LGM_ERR_UNSUPPORTED: return "unsupported";
    case LGM_ERR_STATE: return "invalid state";
    default: return "unknown status";
    }
}

void lgm_config_default(lgm_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    // SimulationParameters() defaults (parameters.h:285-378)
    cfg->grid_x = 128; cfg->grid_y = 128; cfg->grid_z = 1;
    cfg->electrostatic_cutoff = 50;
    // setCalculatedValues (parameters.h:384-390) with the constants of
    // parameters.h:358-362 and dielectric.constant 3.5.
    const double e = 1.60217646e-19, eps0 = 8.854187817e-12, a = 1e-9, epsr = 3.5;
    cfg->electrostatic_prefactor = e / (4.0 * M_PI * epsr * eps0 * a);
    cfg->coulomb_gaussian_sigma = 0.0;
    cfg->work_x = cfg->work_y = cfg->work_z = 4;
    cfg->work_size = 256;
    cfg->opencl_threshold = 256;
    cfg->max_charges = 0;
    cfg->max_targets = 0;
    cfg->precision = LGM_PREC_FP32C;
    cfg->path = LGM_PATH_RSQRT;
}

lgm_status lgm_create(const lgm_config* cfg, int32_t device, lgm_ctx** out) {
    g_create_error.clear();
    if (!cfg || !out) {
        g_create_error = "null argument";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    const lgm_config& cf = *cfg;
    if (cf.grid_x < 1 || cf.grid_y < 1 || cf.grid_z < 1) {
        g_create_error = "grid.x, grid.y and grid.z must be >= 1 (parameters.h:403-414)";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    if (cf.electrostatic_cutoff < 1 || cf.electrostatic_cutoff > 1000) {
        g_create_error = "electrostatic.cutoff must be in [1, 1000]";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    if (!(cf.coulomb_gaussian_sigma >= 0) || !std::isfinite(cf.electrostatic_prefactor)) {
        g_create_error = "coulomb.gaussian.sigma must be >= 0 and the prefactor finite";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    if (cf.precision != LGM_PREC_FP32C && cf.precision != LGM_PREC_FP64) {
        g_create_error = "unknown precision";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    if (cf.path != LGM_PATH_RSQRT && cf.path != LGM_PATH_TABLE && cf.path != LGM_PATH_TABLE64) {
        g_create_error = "unknown path";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    // FP32 exactness of r^2 - 1/2 in expanded form: every intermediate a
    // half-integer below 2^22 with the right-image targets at x' < 2X
    // (6 L^2 < 2^22).
    const long long L = std::max<long long>({2LL * cf.grid_x, cf.grid_y, cf.grid_z + 1});
    if (6 * L * L >= (1LL << 22) ||
        (long long)cf.grid_x * cf.grid_y * cf.grid_z + kDrainIds > INT32_MAX) {
        g_create_error = "lattice too large for exact FP32 r^2 (need 6*max(2X,Y,Z+1)^2 < 2^22)";
        return LGM_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
        return LGM_ERR_NO_DEVICE;
    }
    const int dev = device < 0 ? 0 : device;
    if (dev >= ndev) {
        g_create_error = "device id out of range";
        return LGM_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, dev)) != cudaSuccess) {
        g_create_error = std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e);
        return LGM_ERR_NO_DEVICE;
    }
    if (prop.major != 10) {
        g_create_error = "device is not sm_100 (B200); this library is built for sm_100a only";
        return LGM_ERR_NO_DEVICE;
    }
    lgm_ctx* c = new (std::nothrow) lgm_ctx();
    if (!c) {
        g_create_error = "out of host memory";
        return LGM_ERR_INVALID_ARGUMENT;
    }
    c->cfg = cf;
    c->device = dev;
    c->sm_count = prop.multiProcessorCount;
    c->xy = cf.grid_x * cf.grid_y;
    c->volume = c->xy * cf.grid_z;
    auto bail = [&](const char* what, cudaError_t err) {
        g_create_error = std::string(what) + ": " + cudaGetErrorString(err);
        lgm_destroy(c);
        return LGM_ERR_CUDA;
    };
    if ((e = cudaSetDevice(dev)) != cudaSuccess) return bail("cudaSetDevice", e);
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail("cudaStreamCreate", e);
    if ((e = cudaMalloc(&c->d_err, sizeof(unsigned))) != cudaSuccess) return bail("cudaMalloc", e);
    if ((e = cudaMemset(c->d_err, 0, sizeof(unsigned))) != cudaSuccess) return bail("cudaMemset", e);
    if ((e = cudaMallocHost(&c->h_err, sizeof(unsigned))) != cudaSuccess)
        return bail("cudaMallocHost", e);

    // Tables indexed by the integer r^2 (potential.cpp:268-308 restated per r^2):
    //   rtab[k] = 1/sqrt(k) for 0 < k < c^2, 0 at k = 0 and k = c^2 (point, table path);
    //   gauss: gtab[k] = erf(f sqrt(k))/sqrt(k); with the rsqrt path only the
    //   k where it differs from 1/sqrt(k) in FP32 are kept and entry gtab_k
    //   is NaN (the kernel then falls back to 1/r).
    const int c2 = cf.electrostatic_cutoff * cf.electrostatic_cutoff;
    {
        std::vector<float> rt(c2 + 1, 0.f);
        for (int k = 1; k < c2; ++k) rt[k] = (float)(1.0 / std::sqrt((double)k));
        c->rtab_k = c2;
        if ((e = cudaMalloc(&c->d_rtab, rt.size() * sizeof(float))) != cudaSuccess)
            return bail("cudaMalloc", e);
        if ((e = cudaMemcpy(c->d_rtab, rt.data(), rt.size() * sizeof(float),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail("cudaMemcpy", e);
    }
    {
        const double sig = cf.coulomb_gaussian_sigma;
        std::vector<float> gt;
        if (sig > 0) {
            const double f = 1.0 / (std::sqrt(2.0) * sig);
            int kmax = c2;
            if (cf.path == LGM_PATH_RSQRT) {
                // erfc(f sqrt(k)) < 2^-30 beyond kmax: erf rounds to 1 in FP32
                kmax = 1;
                while (kmax < c2 && std::erfc(f * std::sqrt((double)kmax)) >= 0x1p-30) ++kmax;
            }
            gt.assign(kmax + 1, 0.f);
            for (int k = 1; k < kmax; ++k) {
                const double r = std::sqrt((double)k);
                gt[k] = (float)(std::erf(f * r) / r);
            }
            gt[kmax] = cf.path == LGM_PATH_RSQRT ? std::nanf("") : 0.f;
            c->gtab_k = kmax;
        } else {
            gt.assign(2, 0.f);
            c->gtab_k = 0;
        }
        if ((e = cudaMalloc(&c->d_gtab, gt.size() * sizeof(float))) != cudaSuccess)
            return bail("cudaMalloc", e);
        if ((e = cudaMemcpy(c->d_gtab, gt.data(), gt.size() * sizeof(float),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail("cudaMemcpy", e);
    }
    // FP64 tables of the TABLE64 path: w(k) for every integer r^2 = k <= c^2,
    // correctly rounded in IEEE double, 0 at k = 0 and k = c^2.
    if (cf.path == LGM_PATH_TABLE64) {
        std::vector<double> rt(c2 + 1, 0.0), gt(c2 + 1, 0.0);
        const double sig = cf.coulomb_gaussian_sigma;
        const double f = sig > 0 ? 1.0 / (std::sqrt(2.0) * sig) : 0.0;
        for (int k = 1; k < c2; ++k) {
            const double r = std::sqrt((double)k);
            rt[k] = 1.0 / r;
            gt[k] = sig > 0 ? std::erf(f * r) / r : rt[k];
        }
        if ((e = cudaMalloc(&c->d_rtab64, rt.size() * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&c->d_gtab64, gt.size() * sizeof(double))) != cudaSuccess)
            return bail("cudaMalloc", e);
        if ((e = cudaMemcpy(c->d_rtab64, rt.data(), rt.size() * sizeof(double),
                            cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(c->d_gtab64, gt.data(), gt.size() * sizeof(double),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail("cudaMemcpy", e);
    }
    // Lattice cells for the spatial target order (Morton rank per cell).
    {
        const std::vector<int32_t> rank =
            cell_ranks(cf.grid_x, cf.grid_y, cf.grid_z, &c->cell_shift, &c->cells_x, &c->cells_y);
        c->ncells = (int)rank.size();
        c->bins_stride = (c->ncells + 2 + 3) / 4 * 4;
        if ((e = cudaMalloc(&c->d_cell_rank, sizeof(int32_t) * rank.size())) != cudaSuccess ||
            (e = cudaMalloc(&c->d_bins, sizeof(int32_t) * (2 * c->bins_stride + 4))) !=
                cudaSuccess ||
            (e = cudaMalloc(&c->d_item_count, 3 * sizeof(int32_t))) != cudaSuccess ||
            (e = cudaMalloc(&c->d_cost_hist, kCostBuckets * sizeof(int32_t))) != cudaSuccess)
            return bail("cudaMalloc", e);
        // the source bins follow the target bins, 16-byte aligned (the scan reads int4)
        c->d_sbins = c->d_bins + c->bins_stride;
        if ((e = cudaMemcpy(c->d_cell_rank, rank.data(), sizeof(int32_t) * rank.size(),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail("cudaMemcpy", e);
    }
    // Shared memory above the 48 KB default for large cutoffs, and the
    // resident CTAs per SM of every variant (the split count fills
    // kSplitWaves waves of them).
    {
        const int tab_of[4] = {0, c->gtab_k, std::max(c->rtab_k, c->gtab_k), c->rtab_k};
        for (int v = 0; v < kNumVariants; ++v)
            for (int fi = 0; fi < 4; ++fi) {
                if (!kernel_of(kVariants[v], fi)) continue;
                // the table kernels serve only their own path
                if (fi == 2 && cf.path != LGM_PATH_TABLE) continue;
                if (fi == 3 && cf.path != LGM_PATH_TABLE64) continue;
                const size_t smem = variant_smem(kVariants[v], fi, tab_of[fi]);
                if (smem > 48 * 1024) {
                    if (smem > (size_t)prop.sharedMemPerBlockOptin) {
                        g_create_error = "cutoff too large for the shared-memory tables";
                        lgm_destroy(c);
                        return LGM_ERR_UNSUPPORTED;
                    }
                    if ((e = cudaFuncSetAttribute(kernel_of(kVariants[v], fi),
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem)) != cudaSuccess)
                        return bail("cudaFuncSetAttribute", e);
                }
                int bps = 0;
                if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                         &bps, kernel_of(kVariants[v], fi), variant_threads(kVariants[v]),
                         smem)) != cudaSuccess)
                    return bail("cudaOccupancyMaxActiveBlocksPerMultiprocessor", e);
                c->bps[v][fi] = bps;
            }
    }
    *out = c;
    return LGM_OK;
}

lgm_status lgm_destroy(lgm_ctx* c) {
    if (!c) return LGM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* dev_ptrs[] = {c->d_geo,   c->d_qq,         c->d_tgt,        c->d_part,
                        c->d_s,     c->d_q,          c->d_t,          c->d_o,
                        c->d_gtab,  c->d_rtab,       c->d_err,        c->d_cell_rank,
                        c->d_bins,  c->d_key,        c->d_perm,       c->d_ttmp,
                        c->d_skey,  c->d_stmp,       c->d_cbox,       c->d_gbox,
                        c->d_live,  c->d_items,      c->d_tile_first, c->d_tile_items,
                        c->d_item_count, c->d_examined, c->d_rtab64,  c->d_gtab64,
                        c->d_cost_hist,  c->d_order,     c->d_oitems};
    for (void* p : dev_ptrs)
        if (p) cudaFree(p);
    void* host_ptrs[] = {c->h_s, c->h_q, c->h_t, c->h_o, c->h_err};
    for (void* p : host_ptrs)
        if (p) cudaFreeHost(p);
    if (c->ev_pair0) cudaEventDestroy(c->ev_pair0);
    if (c->ev_pair1) cudaEventDestroy(c->ev_pair1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return LGM_OK;
}

const char* lgm_last_error(const lgm_ctx* c) {
    if (!c) return g_create_error.c_str();
    return c->err.c_str();
}

lgm_status lgm_last_launch(lgm_ctx* c, lgm_launch_info* info) {
    if (!c || !info) return LGM_ERR_INVALID_ARGUMENT;
    if (c->timed_pending) {
        LGM_CUDA(c, cudaEventSynchronize(c->ev_pair1));
        float ms = -1.f;
        LGM_CUDA(c, cudaEventElapsedTime(&ms, c->ev_pair0, c->ev_pair1));
        c->last.pair_kernel_ms = ms;
        c->timed_pending = false;
    }
    if (c->count_pending) {
        unsigned long long n = 0;
        LGM_CUDA(c, cudaMemcpy(&n, c->d_examined, sizeof n, cudaMemcpyDeviceToHost));
        c->last.pairs_examined = (int64_t)n;
        c->count_pending = false;
    }
    *info = c->last;
    return LGM_OK;
}

lgm_status lgm_set_counting(lgm_ctx* c, int32_t enable) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    LGM_CUDA(c, cudaSetDevice(c->device));
    if (enable && !c->d_examined)
        LGM_CUDA(c, cudaMalloc(&c->d_examined, sizeof(unsigned long long)));
    c->counting = enable != 0;
    c->count_pending = false;
    return LGM_OK;
}

lgm_status lgm_set_launch_overlap(lgm_ctx* c, int32_t enable) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    c->overlap = enable != 0;
    return LGM_OK;
}

lgm_status lgm_set_timing(lgm_ctx* c, int32_t enable) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    LGM_CUDA(c, cudaSetDevice(c->device));
    if (enable && !c->ev_pair0) {
        LGM_CUDA(c, cudaEventCreate(&c->ev_pair0));
        LGM_CUDA(c, cudaEventCreate(&c->ev_pair1));
    }
    c->timing = enable != 0;
    c->timed_pending = false;
    return LGM_OK;
}

int32_t lgm_variant_count(void) { return kNumVariants; }

lgm_status lgm_variant_info(int32_t v, int32_t* threads, int32_t* target_pairs, int32_t* run) {
    if (v < 0 || v >= kNumVariants) return LGM_ERR_INVALID_ARGUMENT;
    if (threads) *threads = kVariants[v].nt;
    if (target_pairs) *target_pairs = kVariants[v].rp;
    if (run) *run = kVariants[v].sub;
    return LGM_OK;
}

lgm_status lgm_variant_flags(int32_t v, int32_t* flags) {
    if (v < 0 || v >= kNumVariants || !flags) return LGM_ERR_INVALID_ARGUMENT;
    *flags = (kVariants[v].skip ? LGM_VARIANT_WARP_SKIP : 0) |
             (kVariants[v].cull ? LGM_VARIANT_CULLED : 0) |
             (kVariants[v].ws ? LGM_VARIANT_WARP_SPECIALISED : 0);
    return LGM_OK;
}

lgm_status lgm_variant_items(int32_t v, int32_t* chunks_per_item, int32_t* stages) {
    if (v < 0 || v >= kNumVariants) return LGM_ERR_INVALID_ARGUMENT;
    if (chunks_per_item) *chunks_per_item = kVariants[v].cull ? kVariants[v].per_item : 0;
    if (stages) *stages = kVariants[v].ws;
    return LGM_OK;
}

lgm_status lgm_set_variant(lgm_ctx* c, int32_t v) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    if (v < -1 || v >= kNumVariants) return fail(c, LGM_ERR_INVALID_ARGUMENT, "no such variant");
    c->forced_variant = v;
    return LGM_OK;
}

lgm_status lgm_autotune(lgm_ctx* c, lgm_kind kind, uint32_t terms, int32_t n, int32_t t,
                        int32_t* chosen) {
    lgm_status s = check_common(c, kind, terms, n, t);
    if (s != LGM_OK) return s;
    if (n < 1 || t < 1) return fail(c, LGM_ERR_INVALID_ARGUMENT, "autotune needs n, t >= 1");
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    // Synthetic charges of this size: sites spread over the lattice, q = +-1.
    std::vector<int32_t> hs(n), hq(n), ht(t);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    auto next = [&]() { x ^= x << 13; x ^= x >> 7; x ^= x << 17; return x; };
    for (int j = 0; j < n; ++j) { hs[j] = (int32_t)(next() % c->volume); hq[j] = (next() & 1) ? 1 : -1; }
    for (int g = 0; g < t; ++g) ht[g] = (int32_t)(next() % c->volume);
    if ((s = grow_device(c, &c->d_s, &c->s_cap, (size_t)n)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_q, &c->q_cap, (size_t)n)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_t, &c->t_cap, (size_t)t)) != LGM_OK) return s;
    LGM_CUDA(c, cudaMemcpyAsync(c->d_s, hs.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    LGM_CUDA(c, cudaMemcpyAsync(c->d_q, hq.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    LGM_CUDA(c, cudaMemcpyAsync(c->d_t, ht.data(), sizeof(int32_t) * t, cudaMemcpyHostToDevice, st));
    const Shape sh = shape_of(n, t, terms);
    if ((s = prep(c, terms, c->d_s, c->d_q, n, c->d_t, t, 0, sh, st)) != LGM_OK) return s;
    cudaEvent_t e0, e1;
    LGM_CUDA(c, cudaEventCreate(&e0));
    LGM_CUDA(c, cudaEventCreate(&e1));
    int best = kDefaultVariant;
    float best_ms = 1e30f;
    for (int v = 0; v < kNumVariants; ++v) {
        if (c->cfg.path == LGM_PATH_TABLE64 && !kVariants[v].cull) continue;
        int splits;
        if ((s = launch_pair(c, kind, v, sh, st, &splits)) != LGM_OK) break;  // warm
        float ms[3];
        for (int r = 0; r < 3; ++r) {
            cudaEventRecord(e0, st);
            if ((s = launch_pair(c, kind, v, sh, st, &splits)) != LGM_OK) break;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms[r], e0, e1);
        }
        if (s != LGM_OK) break;
        std::sort(ms, ms + 3);
        if (ms[1] < best_ms) { best_ms = ms[1]; best = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != LGM_OK) return s;
    if ((s = check_device_error(c, st)) != LGM_OK) return s;
    c->tune_cache[tune_key(kind, c->cfg.path, sh.t_phys, sh.n_chunks)] = best;
    if (chosen) *chosen = best;
    return LGM_OK;
}

lgm_status lgm_potentials_async(lgm_ctx* c, lgm_kind kind, uint32_t terms,
                                const int32_t* d_src_site, const int32_t* d_src_q, int32_t n,
                                const int32_t* d_tgt_site, int32_t t, double* d_out,
                                void* stream) {
    lgm_status s = check_common(c, kind, terms, n, t);
    if (s != LGM_OK) return s;
    if ((n > 0 && (!d_src_site || !d_src_q)) || (t > 0 && (!d_tgt_site || !d_out)))
        return fail(c, LGM_ERR_INVALID_ARGUMENT, "null buffer");
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return launch_potentials(c, kind, terms, d_src_site, d_src_q, n, d_tgt_site, t, 0, d_out, st);
}

lgm_status lgm_sync(lgm_ctx* c, void* stream) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return check_device_error(c, st);
}

lgm_status lgm_potentials(lgm_ctx* c, lgm_kind kind, uint32_t terms, const int32_t* src_site,
                          const int32_t* src_q, int32_t n, const int32_t* tgt_site, int32_t t,
                          double* out) {
    lgm_status s = check_common(c, kind, terms, n, t);
    if (s != LGM_OK) return s;
    if ((n > 0 && (!src_site || !src_q)) || (t > 0 && (!tgt_site || !out)))
        return fail(c, LGM_ERR_INVALID_ARGUMENT, "null buffer");
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    if (t == 0) return check_sites(c, src_site, n, nullptr, 0);
    // One pinned staging buffer and one device buffer, laid out [targets t]
    // [charges n][sources n, unless they are the first n targets], cross in
    // one copy; the results come back in one copy with the device error word
    // behind them (written by the call's last kernel).
    const bool alias = tgt_site == src_site && n <= t;
    const size_t words = (size_t)t + n + (alias ? 0 : n);
    if ((s = grow_host(c, &c->h_t, &c->ht_cap, words)) != LGM_OK) return s;
    if ((s = grow_host(c, &c->h_o, &c->ho_cap, (size_t)t + 1)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_t, &c->t_cap, words)) != LGM_OK) return s;
    if ((s = grow_device(c, &c->d_o, &c->o_cap, (size_t)t + 1)) != LGM_OK) return s;
    // The sites are checked on the device (prep_records), which gives each an
    // empty record and raises an error bit; only then are they checked here,
    // for the first bad one (sources first, then targets, as check_sites
    // reports them).  When the sources are the first n targets (kernel 2: w
    // aliases s, openclhelper.cpp:154) they cross once, as targets.
    std::memcpy(c->h_t, tgt_site, sizeof(int32_t) * t);
    if (n > 0) std::memcpy(c->h_t + t, src_q, sizeof(int32_t) * n);
    if (!alias && n > 0) std::memcpy(c->h_t + t + n, src_site, sizeof(int32_t) * n);
    LGM_CUDA(c, cudaMemcpyAsync(c->d_t, c->h_t, sizeof(int32_t) * words, cudaMemcpyHostToDevice,
                                st));
    const int32_t* d_src = alias ? c->d_t : c->d_t + t + n;
    unsigned* d_err_out = reinterpret_cast<unsigned*>(c->d_o + t);
    if ((s = launch_potentials(c, kind, terms, d_src, c->d_t + t, n, c->d_t, t, 0, c->d_o, st,
                               d_err_out)) != LGM_OK)
        return s;
    LGM_CUDA(c, cudaMemcpyAsync(c->h_o, c->d_o, sizeof(double) * ((size_t)t + 1),
                                cudaMemcpyDeviceToHost, st));
    LGM_CUDA(c, cudaStreamSynchronize(st));
    const unsigned e = *reinterpret_cast<const unsigned*>(c->h_o + t);
    if (e != 0) {
        const lgm_status ds = device_error_status(c, st, e);  // clears the device word
        if (e & (DEVERR_SOURCE_RANGE | DEVERR_TARGET_RANGE)) {
            const lgm_status hs = check_sites(c, src_site, n, tgt_site, t);
            if (hs != LGM_OK) return hs;
        }
        return ds;
    }
    std::memcpy(out, c->h_o, sizeof(double) * t);
    return LGM_OK;
}

lgm_status lgm_coulomb_kernel2(lgm_ctx* c, lgm_kind kind, const int32_t* s, const int32_t* q,
                               int32_t n, int32_t total, double* o) {
    if (c && (n < 0 || n > total)) return fail(c, LGM_ERR_INVALID_ARGUMENT, "need 0 <= n <= total");
    // kernel 2: w aliases s (openclhelper.cpp:154), the first n entries are
    // the sources, every entry is a target.
    return lgm_potentials(c, kind, LGM_TERM_DIRECT, s, q, n, s, total, o);
}

lgm_status lgm_coulomb_kernel1_async(lgm_ctx* c, lgm_kind kind, const int32_t* d_s,
                                     const int32_t* d_q, int32_t n, double* d_o, void* stream) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    lgm_status st = check_common(c, kind, LGM_TERM_DIRECT, n, 0);
    if (st != LGM_OK) return st;
    if ((n > 0 && (!d_s || !d_q)) || !d_o) return fail(c, LGM_ERR_INVALID_ARGUMENT, "null buffer");
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    return launch_potentials(c, kind, LGM_TERM_DIRECT, d_s, d_q, n, nullptr, c->volume, 1, d_o, s);
}

lgm_status lgm_coulomb_kernel1(lgm_ctx* c, lgm_kind kind, const int32_t* s, const int32_t* q,
                               int32_t n, double* o) {
    if (!c) return LGM_ERR_INVALID_ARGUMENT;
    lgm_status st = check_common(c, kind, LGM_TERM_DIRECT, n, 0);
    if (st != LGM_OK) return st;
    if ((n > 0 && (!s || !q)) || !o) return fail(c, LGM_ERR_INVALID_ARGUMENT, "null buffer");
    if ((st = check_sites(c, s, n, nullptr, 0)) != LGM_OK) return st;
    LGM_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t str = c->stream;
    const size_t nn = std::max(n, 1);
    const size_t vv = (size_t)c->volume;
    if ((st = grow_host(c, &c->h_s, &c->hs_cap, nn)) != LGM_OK) return st;
    if ((st = grow_host(c, &c->h_q, &c->hq_cap, nn)) != LGM_OK) return st;
    if ((st = grow_host(c, &c->h_o, &c->ho_cap, vv)) != LGM_OK) return st;
    if ((st = grow_device(c, &c->d_s, &c->s_cap, nn)) != LGM_OK) return st;
    if ((st = grow_device(c, &c->d_q, &c->q_cap, nn)) != LGM_OK) return st;
    if ((st = grow_device(c, &c->d_o, &c->o_cap, vv)) != LGM_OK) return st;
    std::memcpy(c->h_s, s, sizeof(int32_t) * n);
    std::memcpy(c->h_q, q, sizeof(int32_t) * n);
    LGM_CUDA(c, cudaMemcpyAsync(c->d_s, c->h_s, sizeof(int32_t) * n, cudaMemcpyHostToDevice, str));
    LGM_CUDA(c, cudaMemcpyAsync(c->d_q, c->h_q, sizeof(int32_t) * n, cudaMemcpyHostToDevice, str));
    if ((st = launch_potentials(c, kind, LGM_TERM_DIRECT, c->d_s, c->d_q, n, nullptr, c->volume, 1,
                                c->d_o, str)) != LGM_OK)
        return st;
    LGM_CUDA(c, cudaMemcpyAsync(c->h_o, c->d_o, sizeof(double) * vv, cudaMemcpyDeviceToHost, str));
    if ((st = check_device_error(c, str)) != LGM_OK) return st;
    std::memcpy(o, c->h_o, sizeof(double) * vv);
    return LGM_OK;
}

}  // extern "C"
