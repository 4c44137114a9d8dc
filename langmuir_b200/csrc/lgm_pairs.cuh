// lgm_pairs.cuh -- the all-pairs Coulomb sum on sm_100a.
//
// Replaces the reference's coulomb2/gauss2 (and coulomb1/gauss1) OpenCL
// kernels (src/langmuirCore/kernel.cl:56-369): for every target site the sum
// over all source charges of q_j w(r), 0 < r^2 < cutoff^2.
//
// Layout (built by the prep kernels in lgm_api.cu):
//   source j  -> two float4 {a,a,b,b},{c,c,d,d} with a,b,c = -2x,-2y,-2z and
//                d = x^2+y^2+z^2 - 1/2, and one float2 {q,q};
//   target p  -> float4 {x, y, z, x^2+y^2+z^2}.
// Then u = d + tt + x*a + y*b + z*c = r^2 - 1/2: one add and three FMAs,
// every intermediate a half-integer below 2^22, so u is exact in FP32.  Each
// component is stored twice so that one packed FP32x2 instruction serves two
// targets of a thread.
//
// Per pair:  u = r^2 - 1/2 (exact), r^2 = u + 1/2, y = rsqrt(r^2) (MUFU) and,
// predicated on 0 < u < c^2 - 1/2, acc += q * y.  The predicate is one
// unsigned compare of u's bit pattern (negative u has the sign bit set, so
// r = 0 fails it as r^2 >= c^2 does): the cutoff and the reference's r = 0
// skip cost one ALU instruction, and the accumulate is a predicated FFMA.
// Accumulation: runs of SUB sources in FP32, each run folded into an FP64
// accumulator per target; split partials summed in FP64 in a fixed order.
//
// Sources are staged through shared memory in chunks of CH by bulk TMA copies
// (cp.async.bulk, no multicast) on two mbarrier-tracked stages; all threads
// read each source by broadcast.
//
// SKIP tiles run on targets in spatial order (the host sorts them by lattice
// cell): a warp owns 64*RP consecutive targets, which lie close together.
// Every pair's r^2 is still computed and tested; when no pair of the warp's
// targets with a source is inside the cutoff, the warp skips that source's
// rsqrt and accumulation (a warp vote).  Skipped pairs would have added
// nothing, so the sums are bit for bit those of the plain tile.
#pragma once

#include <algorithm>
#include <utility>
#include <vector>

#include "lgm_device.cuh"

namespace lgm {

constexpr int CH = 128;   // sources per shared-memory stage

struct PairArgs {
    const float4* geo = nullptr;      // [n_pad * 2]
    const float2* qq = nullptr;       // [n_pad]
    int n_chunks = 0;                 // n_pad / CH
    int splits = 1;                   // source splits (gridDim.y)
    const float4* tgt = nullptr;      // [t_phys]
    int t_phys = 0;                   // physical targets (padded)
    double* part = nullptr;           // [splits][t_phys]
    float c2 = 0.f;                   // cutoff^2
    const float* tab = nullptr;       // gauss correction table or 1/sqrt(k) table
    const double* tab64 = nullptr;    // FP64 w(k) for every integer r^2 = k (TABLE64 path)
    int tab_k = 0;                    // last valid table index (clamp)
    unsigned* err = nullptr;
    // Optional: counts read on the device (dyn[0] = n_chunks, dyn[1] = t_phys)
    // so one launch shape serves every step of a simulation.
    const int* dyn = nullptr;
    // NORM kernels: sum over FP32 runs of |run sum| per target.  When every
    // run holds charges of one sign (charge classes padded to whole chunks)
    // this is prefactor-free N = sum_j |q_j| w(r_j), the error scale of the
    // target's potential.  Layout [splits][t_phys].
    float* part_norm = nullptr;
};

// Kernel launched with dynamic shared memory pair_smem_bytes(tab_k).
__host__ __device__ constexpr size_t pair_stage_bytes() {
    return (size_t)CH * (2 * sizeof(float4) + sizeof(float2));
}
inline size_t pair_smem_bytes(int tab_k) {
    return 2 * pair_stage_bytes() + 16 + (size_t)(tab_k + 1) * sizeof(float) + 16;
}
// The same with the FP64 table of the TABLE64 path (PATH 2).
inline size_t pair_smem_bytes64(int tab_k) {
    return 2 * pair_stage_bytes() + 16 + (size_t)(tab_k + 1) * sizeof(double) + 16;
}

// KIND 0 point, 1 gauss.  PATH 0 MUFU rsqrt, 1 shared-memory table of w(k)
// for every integer r^2 = k (entries 0 and c^2 are 0).  NT threads, RP target
// pairs per thread, SUB sources per FP32 run (SUB divides CH).
// One CTA's work: target tile `tile`, source split `split` of A.splits.
template <int KIND, int PATH, int NT, int RP, int SUB, bool NORM, bool SKIP = false>
__device__ __forceinline__ void pair_tile(PairArgs A, const int tile, const int split) {
    static_assert(!SKIP || PATH == 0, "the warp skip serves the rsqrt path");
    static_assert(CH % SUB == 0, "SUB must divide CH");
    if (A.dyn) {
        A.n_chunks = A.dyn[0];
        A.t_phys = A.dyn[1];
    }
    if (tile * (NT * 2 * RP) >= A.t_phys) return;  // tile beyond this launch's targets
    extern __shared__ __align__(128) unsigned char smem[];
    float4* s_geo = reinterpret_cast<float4*>(smem);                       // [2][CH*2]
    float2* s_qq = reinterpret_cast<float2*>(smem + 2 * CH * 2 * sizeof(float4));  // [2][CH]
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem + 2 * pair_stage_bytes());
    float* s_tab = reinterpret_cast<float*>(smem + 2 * pair_stage_bytes() + 16);

    const int tid = threadIdx.x;
    const int c_begin = (int)((long long)split * A.n_chunks / A.splits);
    const int c_end = (int)((long long)(split + 1) * A.n_chunks / A.splits);
    const int nck = c_end - c_begin;

    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_mbar_init();
    }
    if (KIND == 1 || PATH == 1)
        for (int k = tid; k <= A.tab_k; k += NT) s_tab[k] = A.tab[k];
    __syncthreads();

    auto issue = [&](int i) {
        const int st = i & 1;
        const int chunk = c_begin + i;
        mbar_arrive_expect_tx(&s_bar[st], (uint32_t)pair_stage_bytes());
        bulk_g2s(s_geo + st * CH * 2, A.geo + (size_t)chunk * CH * 2,
                 (uint32_t)(CH * 2 * sizeof(float4)), &s_bar[st]);
        bulk_g2s(s_qq + st * CH, A.qq + (size_t)chunk * CH, (uint32_t)(CH * sizeof(float2)),
                 &s_bar[st]);
    };
    if (tid == 0) {
        if (nck > 0) issue(0);
        if (nck > 1) issue(1);
    }

    // Targets of this thread: p = base + tid + k*NT, k = 0 .. 2*RP-1 (SKIP:
    // p = base + warp*64*RP + k*32 + lane); pair k packs targets 2k and 2k+1.
    const int base = tile * (NT * 2 * RP);
    auto target_of = [&](int k) {
        return SKIP ? base + (tid >> 5) * (64 * RP) + k * 32 + (tid & 31) : base + tid + k * NT;
    };
    float2 tx[RP], ty[RP], tz[RP], tt[RP];
#pragma unroll
    for (int k = 0; k < RP; ++k) {
        const int p0 = target_of(2 * k);
        const int p1 = target_of(2 * k + 1);
        const float4 a = p0 < A.t_phys ? A.tgt[p0] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 b = p1 < A.t_phys ? A.tgt[p1] : make_float4(0.f, 0.f, 0.f, 0.f);
        tx[k] = f2(a.x, b.x); ty[k] = f2(a.y, b.y); tz[k] = f2(a.z, b.z); tt[k] = f2(a.w, b.w);
    }
    double acc64[2 * RP];
    float nrm[NORM ? 2 * RP : 1];
#pragma unroll
    for (int k = 0; k < 2 * RP; ++k) acc64[k] = 0.0;
#pragma unroll
    for (int k = 0; k < (NORM ? 2 * RP : 1); ++k) nrm[k] = 0.f;
    const unsigned ulim = __float_as_uint(A.c2 - 0.5f);
    const float2 half2 = f2(0.5f, 0.5f);

    int failed_at = -1;

    for (int i = 0; i < nck; ++i) {
        const int st = i & 1;
        const uint32_t parity = (uint32_t)((i >> 1) & 1);
        bool mine = mbar_wait_bounded(&s_bar[st], parity, A.err);
        if (!__syncthreads_and(mine)) { failed_at = i; break; }
        const float4* sg = s_geo + st * CH * 2;
        const float2* sq = s_qq + st * CH;

#pragma unroll 1
        for (int j0 = 0; j0 < CH; j0 += SUB) {
            float acc[2 * RP];
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) acc[k] = 0.f;
            // the skip tile branches per source: a partial unroll keeps its code small
            constexpr int kUnrollJ = SKIP ? 4 : SUB;
#pragma unroll kUnrollJ
            for (int jj = 0; jj < SUB; ++jj) {
                const int j = j0 + jj;
                const float4 g0 = sg[2 * j];
                const float4 g1 = sg[2 * j + 1];
                const float2 av = f2(g0.x, g0.y), bv = f2(g0.z, g0.w);
                const float2 cv = f2(g1.x, g1.y), dv = f2(g1.z, g1.w);
                if constexpr (SKIP) {
                    // r^2 - 1/2 as (tt + x a) + y b + (d + z c): three
                    // dependent steps instead of four.  Every partial sum is
                    // an integer or half-integer no larger in magnitude than
                    // |t|^2 + |s|^2, so each step is exact and u has the bits
                    // of the plain tile's order.  The per-thread minimum is a
                    // tree for the same reason.
                    float2 uu[RP];
                    unsigned mk[RP];
#pragma unroll
                    for (int k = 0; k < RP; ++k) {
                        const float2 pa = __ffma2_rn(tx[k], av, tt[k]);
                        const float2 pc = __ffma2_rn(tz[k], cv, dv);
                        uu[k] = __fadd2_rn(__ffma2_rn(ty[k], bv, pa), pc);
                        mk[k] = min(__float_as_uint(uu[k].x), __float_as_uint(uu[k].y));
                    }
#pragma unroll
                    for (int w = 1; w < RP; w *= 2)
#pragma unroll
                        for (int k = 0; k + w < RP; k += 2 * w) mk[k] = min(mk[k], mk[k + w]);
                    const unsigned m = mk[0];
                    if (__any_sync(0xffffffffu, m < ulim)) {
                        const float qs = sq[j].x;
#pragma unroll
                        for (int k = 0; k < RP; ++k) {
                            const float2 r2 = __fadd2_rn(uu[k], half2);
                            float wx = rsqrt_mufu(r2.x);
                            float wy = rsqrt_mufu(r2.y);
                            if (KIND == 1) {
                                const int ix =
                                    min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, A.tab_k);
                                const int iy =
                                    min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, A.tab_k);
                                wx = fminf(s_tab[ix], wx);
                                wy = fminf(s_tab[iy], wy);
                            }
                            fma_if_below(acc[2 * k], qs, wx, __float_as_uint(uu[k].x), ulim);
                            fma_if_below(acc[2 * k + 1], qs, wy, __float_as_uint(uu[k].y), ulim);
                        }
                    }
                    continue;
                }
                const float qs = sq[j].x;
#pragma unroll
                for (int k = 0; k < RP; ++k) {
                    float2 u = __fadd2_rn(dv, tt[k]);
                    u = __ffma2_rn(tx[k], av, u);
                    u = __ffma2_rn(ty[k], bv, u);
                    u = __ffma2_rn(tz[k], cv, u);  // r^2 - 1/2, exact
                    const float2 r2 = __fadd2_rn(u, half2);
                    float wx, wy;
                    if (PATH == 1) {
                        // w(k) from the table; entries 0 and c^2 are 0, so the
                        // clamp also applies the cutoff and the r = 0 skip.
                        const int ix = min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, A.tab_k);
                        const int iy = min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, A.tab_k);
                        wx = s_tab[ix];
                        wy = s_tab[iy];
                    } else {
                        wx = rsqrt_mufu(r2.x);
                        wy = rsqrt_mufu(r2.y);
                        if (KIND == 1) {
                            // erf(f r)/r: the tabulated value for r^2 < tab_k,
                            // else 1/r (entry tab_k is NaN: fminf returns 1/r).
                            const int ix =
                                min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, A.tab_k);
                            const int iy =
                                min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, A.tab_k);
                            wx = fminf(s_tab[ix], wx);
                            wy = fminf(s_tab[iy], wy);
                        }
                    }
                    fma_if_below(acc[2 * k], qs, wx, __float_as_uint(u.x), ulim);
                    fma_if_below(acc[2 * k + 1], qs, wy, __float_as_uint(u.y), ulim);
                }
            }
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) acc64[k] += (double)acc[k];
            if (NORM) {
#pragma unroll
                for (int k = 0; k < 2 * RP; ++k) nrm[NORM ? k : 0] += fabsf(acc[k]);
            }
        }
        __syncthreads();  // every thread is done with stage st
        if (tid == 0 && i + 2 < nck) {
            fence_proxy_async_smem();
            issue(i + 2);
        }
    }

    if (failed_at >= 0) {
        // A stage never completed: wait (bounded) for the copies this CTA
        // still has in flight -- chunks failed_at and failed_at + 1 -- then
        // leave without writing results; the host sees DEVERR_TIMEOUT.
        if (tid == 0)
            mbar_drain_stages(s_bar, (uint32_t)failed_at, (uint32_t)min(failed_at + 2, nck));
        return;
    }

    double* out = A.part + (size_t)split * A.t_phys;
#pragma unroll
    for (int k = 0; k < 2 * RP; ++k) {
        const int p = target_of(k);
        if (p < A.t_phys) {
            out[p] = acc64[k];
            if (NORM) A.part_norm[(size_t)split * A.t_phys + p] = nrm[NORM ? k : 0];
        }
    }
}

// Grid form: blockIdx.x = target tile, blockIdx.y = source split.
template <int KIND, int PATH, int NT, int RP, int SUB, bool NORM = false, bool SKIP = false>
__global__ void __launch_bounds__(NT) pair_kernel(PairArgs A) {
    pdl_wait();
    pdl_trigger();
    pair_tile<KIND, PATH, NT, RP, SUB, NORM, SKIP>(A, blockIdx.x, blockIdx.y);
}

// Work-item form for many independent problems in one launch (batched
// replicas): item = {problem, tile, split, splits}; problem p's arguments are
// args[p].  Items of uneven problems share the grid.
template <int KIND, int PATH, int NT, int RP, int SUB, bool NORM = false, bool SKIP = false>
__global__ void __launch_bounds__(NT) pair_kernel_items(const PairArgs* __restrict__ args,
                                                        const int4* __restrict__ items) {
    const int4 it = items[blockIdx.x];
    PairArgs A = args[it.x];
    A.splits = it.w;
    pair_tile<KIND, PATH, NT, RP, SUB, NORM, SKIP>(A, it.y, it.z);
}

// Exclusive prefix sum of a[0..n) in place by one block (blockDim a multiple
// of 32, at most 1024; every thread of the block calls it; a 16-byte
// aligned).  Each thread owns a run of consecutive entries, a multiple of 4
// long, read and written as int4 so that its loads are in flight together.
__device__ __forceinline__ void block_exclusive_scan(int32_t* a, int n) {
    __shared__ int32_t warp_tot[32];
    const int nt = (int)blockDim.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = ((n + nt - 1) / nt + 3) & ~3;
    const int lo = min(n, tid * per), hi = min(n, lo + per);
    const int hi4 = lo + ((hi - lo) & ~3);
    int32_t sum = 0;
#pragma unroll 4
    for (int i = lo; i < hi4; i += 4) {
        const int4 q = *reinterpret_cast<const int4*>(a + i);
        sum += q.x + q.y + q.z + q.w;
    }
    for (int i = hi4; i < hi; ++i) sum += a[i];
    int32_t incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int32_t w = lane < nt / 32 ? warp_tot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += v;
        }
        if (lane < nt / 32) warp_tot[lane] = w;
    }
    __syncthreads();
    int32_t run = incl - sum + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll 4
    for (int i = lo; i < hi4; i += 4) {
        int4 q = *reinterpret_cast<int4*>(a + i);
        const int4 c = q;
        q.x = run; run += c.x;
        q.y = run; run += c.y;
        q.z = run; run += c.z;
        q.w = run; run += c.w;
        *reinterpret_cast<int4*>(a + i) = q;
    }
    for (int i = hi4; i < hi; ++i) {
        const int32_t c = a[i];
        a[i] = run;
        run += c;
    }
    __syncthreads();
}

// Morton (Z-order) rank of every lattice cell -- cubes of 2^shift sites, the
// shift the smallest from 3 up that keeps the cells at most 65536 -- for
// sorting targets and sources in spatial order.  Cells of 8^3 sites rather
// than 4^3 cut the bins (and the scans over them) eightfold for a slightly
// coarser order: on 256x256x16 with 2% charges the culled sums examine 0.4%
// more pairs.  Host side; returns the rank table.
inline std::vector<int32_t> cell_ranks(int X, int Y, int Z, int* shift, int* cx, int* cy) {
    int sh = 3;
    auto cells = [&](int d) { return (d + (1 << sh) - 1) >> sh; };
    while ((long long)cells(X) * cells(Y) * cells(Z) > 65536) ++sh;
    *shift = sh;
    *cx = cells(X);
    *cy = cells(Y);
    const int cz = cells(Z);
    const int n = *cx * *cy * cz;
    auto spread = [](uint64_t v) {  // bit i of v to bit 3i
        uint64_t r = 0;
        for (int i = 0; i < 21; ++i) r |= ((v >> i) & 1ull) << (3 * i);
        return r;
    };
    std::vector<std::pair<uint64_t, int>> code(n);
    for (int z = 0; z < cz; ++z)
        for (int y = 0; y < *cy; ++y)
            for (int x = 0; x < *cx; ++x) {
                const int cell = x + *cx * (y + *cy * z);
                code[cell] = {spread(x) | (spread(y) << 1) | (spread(z) << 2), cell};
            }
    std::sort(code.begin(), code.end());
    std::vector<int32_t> rank(n);
    for (int r = 0; r < n; ++r) rank[code[r].second] = r;
    return rank;
}

}  // namespace lgm
