// lgm_cull.cuh -- the pair sum over spatially culled source chunks.
//
// The reference's coulomb2/gauss2 (src/langmuirCore/kernel.cl:222-369) test
// every (target, source) pair against the cutoff.  With the sources in
// spatial order (sorted by lattice cell) and the targets too, whole blocks of
// pairs lie beyond the cutoff and add exactly nothing, so they need not be
// visited at all:
//
//   chunk_boxes  the bounding box of every source chunk (CH = 128 sources)
//                and of each of its eight groups of 16;
//   cull         per target tile (the targets of one CTA), the ordered list
//                of source chunks whose box comes within the cutoff of the
//                tile's box, cut into work items of at most `per_item` chunks;
//   pair         a persistent kernel: CTA b takes items b, b + G, b + 2G, ...
//                and streams their chunks through shared memory (bulk TMA, two
//                stages, the next item's chunks prefetched across the item
//                boundary).  Each warp skips a 16-source group whose box lies
//                beyond the cutoff of its own targets' box, and inside a live
//                group the warp still votes per source (the SKIP tile of
//                lgm_pairs.cuh);
//   finalize     per target, the partials of its tile's items summed in item
//                (= chunk) order.
//
// A skipped chunk or group holds only pairs with r^2 >= c^2 (box distance
// tested exactly in integers), whose terms are zero; an FP32 run over a
// skipped group would have summed to +0 and been folded as a no-op.  The sums
// are therefore those of the unculled tile over the same source order, and
// they are deterministic: items of a tile are numbered in chunk order, and a
// tile's partials are added in that order whatever CTA computed them.
#pragma once

#include "lgm_pairs.cuh"

namespace lgm {

constexpr int kGroup = 16;                    // sources per group box
constexpr int kGroupsPerChunk = CH / kGroup;  // 8
constexpr int kCullThreads = 256;             // threads of the cull kernel
constexpr int kMaxItemsPerTile = 32;          // items a tile's chunk list is cut into, at most
constexpr int kMaxSegments = 16;              // warp target segments of a tile, at most
constexpr int kCostBuckets = 256;             // item cost classes of the largest-first order
constexpr int kLiveSmem = 1024;               // live chunks the cull keeps in shared memory

// A box of lattice coordinates [lo, hi] per axis (inclusive).  Empty: lo > hi.
struct __align__(16) Box {
    short xl, yl, zl, pad0;
    short xh, yh, zh, pad1;
};

__host__ __device__ inline Box empty_box() {
    Box b;
    b.xl = b.yl = b.zl = 32767;
    b.xh = b.yh = b.zh = -32768;
    b.pad0 = b.pad1 = 0;
    return b;
}

// Squared distance between two boxes (0 when they overlap); each axis gap is
// clamped at 4096 so that empty boxes give a large value without overflow.
__device__ __forceinline__ int box_gap2(const Box& a, const Box& b) {
    const int gx = min(4096, max(0, max(a.xl - b.xh, b.xl - a.xh)));
    const int gy = min(4096, max(0, max(a.yl - b.yh, b.yl - a.yh)));
    const int gz = min(4096, max(0, max(a.zl - b.zh, b.zl - a.zh)));
    return gx * gx + gy * gy + gz * gz;
}

// Min and max of six coordinates over a full warp.
__device__ __forceinline__ void warp_box(int& xl, int& yl, int& zl, int& xh, int& yh, int& zh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        xl = min(xl, __shfl_xor_sync(0xffffffffu, xl, o));
        yl = min(yl, __shfl_xor_sync(0xffffffffu, yl, o));
        zl = min(zl, __shfl_xor_sync(0xffffffffu, zl, o));
        xh = max(xh, __shfl_xor_sync(0xffffffffu, xh, o));
        yh = max(yh, __shfl_xor_sync(0xffffffffu, yh, o));
        zh = max(zh, __shfl_xor_sync(0xffffffffu, zh, o));
    }
}

__device__ __forceinline__ Box make_box(int xl, int yl, int zl, int xh, int yh, int zh) {
    Box b;
    b.xl = (short)max(xl, -32768); b.yl = (short)max(yl, -32768); b.zl = (short)max(zl, -32768);
    b.xh = (short)min(xh, 32767);  b.yh = (short)min(yh, 32767);  b.zh = (short)min(zh, 32767);
    b.pad0 = b.pad1 = 0;
    return b;
}

struct CullArgs {
    // sources (records as PairArgs) and their boxes
    int n_chunks = 0;                 // source chunks (dyn[0] overrides)
    Box* cbox = nullptr;              // [chunks]
    Box* gbox = nullptr;              // [chunks * kGroupsPerChunk]
    // targets
    const float4* tgt = nullptr;      // physical target records (w < 0: padding)
    int t_phys = 0;                   // physical targets (dyn[1] overrides)
    const int* dyn = nullptr;         // as PairArgs::dyn
    int c2 = 0;                       // cutoff^2
    int tile_size = 0;                // targets per tile = NT * 2 * RP of the pair kernel
    // the work list
    int per_item = 2;                 // chunks per item (fewer items are never cut)
    int max_items = kMaxItemsPerTile; // items per tile, at most
    int32_t* live = nullptr;          // [tiles][live_stride] live chunk ids in order
    int live_stride = 0;
    int4* items = nullptr;            // {tile, first live index, chunk count, 0}
    int* item_count = nullptr;        // items written (zeroed by chunk_boxes block 0)
    int* work = nullptr;              // next item to take, warp-specialised kernel (zeroed
                                      // by chunk_boxes block 0; may be null otherwise)
    int* tile_first = nullptr;        // [tiles] first item of the tile
    int* tile_items = nullptr;        // [tiles] items of the tile
    // Optional (null: off): pairs whose r^2 the pair kernel computed, i.e.
    // 32 sources x 64 RP targets per live group of a warp, summed over warps.
    unsigned long long* examined = nullptr;
    // Optional largest-first order (hist null: off).  warp_targets: targets
    // of one warp of the pair kernel (64 RP); an item's cost is the number of
    // (warp, group) pairs whose boxes lie within the cutoff, i.e. the groups
    // the pair kernel's warps will visit; hist[kCostBuckets] counts items per
    // cost (zeroed by chunk_boxes block 0), and order_items writes order[]:
    // the items by decreasing cost, which the pair kernels take in turn.
    int warp_targets = 0;
    int* hist = nullptr;
    int* order = nullptr;
    // Optional with order: the item records in order[]'s order, .w = the
    // item's index (one load fewer for the kernels that take items in turn)
    int4* oitems = nullptr;
    // with order: culled tiles so far (zeroed by chunk_boxes block 0); the
    // cull's last block to finish writes order[]
    int* done = nullptr;
};

// One block of CH threads per source chunk: group (kGroup) and chunk boxes of the
// records with a nonzero charge.  Block 0 also zeroes the item counter for
// the cull that follows.
__device__ __forceinline__ void chunk_boxes_body(const PairArgs& A, const CullArgs& C,
                                                 const int chunk) {
    __shared__ Box s_g[kGroupsPerChunk];
    const int n_chunks = A.dyn ? A.dyn[0] : A.n_chunks;
    if (chunk == 0) {
        if (threadIdx.x == 0) {
            if (C.item_count) *C.item_count = 0;
            if (C.work) *C.work = 0;
            if (C.done) *C.done = 0;
        }
        if (C.hist)
            for (int b = (int)threadIdx.x; b < kCostBuckets; b += (int)blockDim.x) C.hist[b] = 0;
    }
    if (chunk >= n_chunks) return;
    const int j = chunk * CH + (int)threadIdx.x;
    const float4 g0 = A.geo[2 * j], g1 = A.geo[2 * j + 1];
    const bool valid = A.qq[j].x != 0.f;
    const int x = (int)(-0.5f * g0.x), y = (int)(-0.5f * g0.z), z = (int)(-0.5f * g1.x);
    int xl = valid ? x : 32767, yl = valid ? y : 32767, zl = valid ? z : 32767;
    int xh = valid ? x : -32768, yh = valid ? y : -32768, zh = valid ? z : -32768;
    // min and max over each aligned group of kGroup lanes
#pragma unroll
    for (int o = kGroup / 2; o > 0; o >>= 1) {
        xl = min(xl, __shfl_xor_sync(0xffffffffu, xl, o));
        yl = min(yl, __shfl_xor_sync(0xffffffffu, yl, o));
        zl = min(zl, __shfl_xor_sync(0xffffffffu, zl, o));
        xh = max(xh, __shfl_xor_sync(0xffffffffu, xh, o));
        yh = max(yh, __shfl_xor_sync(0xffffffffu, yh, o));
        zh = max(zh, __shfl_xor_sync(0xffffffffu, zh, o));
    }
    const int grp = (int)threadIdx.x / kGroup;
    if ((threadIdx.x % kGroup) == 0) {
        const Box b = make_box(xl, yl, zl, xh, yh, zh);
        C.gbox[chunk * kGroupsPerChunk + grp] = b;
        s_g[grp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        Box u = s_g[0];
        for (int g = 1; g < kGroupsPerChunk; ++g) {
            u.xl = min(u.xl, s_g[g].xl); u.yl = min(u.yl, s_g[g].yl); u.zl = min(u.zl, s_g[g].zl);
            u.xh = max(u.xh, s_g[g].xh); u.yh = max(u.yh, s_g[g].yh); u.zh = max(u.zh, s_g[g].zh);
        }
        C.cbox[chunk] = u;
    }
}

// order[] = the items by decreasing cost (a counting sort over the cost
// classes; the order inside a class is arbitrary and changes no sum: an
// item's partials go to its own slot whichever CTA computes it).  One block;
// the reads bypass L1 (the other blocks' writes are in L2).
// s_off[b] = the items of cost classes above b, from the class counts in
// s_off (an exclusive scan in decreasing class order); every thread of a
// block of at least kCostBuckets threads calls it.
__device__ __forceinline__ void cost_offsets(int* s_off) {
    static_assert(kCostBuckets == 256, "one bucket per thread of eight warps");
    __shared__ int s_w[kCostBuckets / 32];
    const int t = (int)threadIdx.x, lane = t & 31;
    const int b = kCostBuckets - 1 - t;  // thread t takes class 255 - t
    const int v = t < kCostBuckets ? s_off[b] : 0;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (t < kCostBuckets && lane == 31) s_w[t >> 5] = inc;
    __syncthreads();
    if (t < kCostBuckets) {
        int before = 0;
        for (int w = 0; w < (t >> 5); ++w) before += s_w[w];
        s_off[b] = before + inc - v;
    }
    __syncthreads();
}

__device__ __forceinline__ void order_items_body(const CullArgs& C) {
    __shared__ int s_off[kCostBuckets];
    const int nit = __ldcg(C.item_count);
    for (int b = (int)threadIdx.x; b < kCostBuckets; b += (int)blockDim.x)
        s_off[b] = __ldcg(&C.hist[b]);
    __syncthreads();
    cost_offsets(s_off);
    const int nt = (int)blockDim.x;
    constexpr int kLoads = 8;  // item loads in flight per thread
    for (int g0 = (int)threadIdx.x; g0 < nit; g0 += kLoads * nt) {
        int4 r[kLoads];
#pragma unroll
        for (int u = 0; u < kLoads; ++u) {
            const int g = g0 + u * nt;
            r[u] = g < nit ? __ldcg(&C.items[g]) : make_int4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < kLoads; ++u) {
            const int g = g0 + u * nt;
            if (g < nit) {
                const int pos = atomicAdd(&s_off[min(r[u].w, kCostBuckets - 1)], 1);
                C.order[pos] = g;
                if (C.oitems) C.oitems[pos] = make_int4(r[u].x, r[u].y, r[u].z, g);
            }
        }
    }
}

// The cull's last block to finish (every block fences its items and costs,
// then counts itself in C.done) writes the order.
__device__ __forceinline__ void cull_last_orders(const CullArgs& C) {
    __shared__ int s_last;
    __syncthreads();  // every thread's items and histogram adds are issued
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(C.done, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    order_items_body(C);
}

// One block of kCullThreads per target tile: the tile's box, its live chunks
// in source order, and its work items.
__device__ __forceinline__ void cull_body(const CullArgs& C, const int tile) {
    __shared__ Box s_seg[kMaxSegments];
    __shared__ int s_wcount[kCullThreads / 32];
    __shared__ int s_cost[kMaxItemsPerTile];
    __shared__ int s_wcost[kMaxItemsPerTile * kMaxSegments];  // per (item, segment) groups
    __shared__ int s_live[kLiveSmem];  // the live list, when it fits
    __shared__ int s_base;
    const int n_chunks = C.dyn ? C.dyn[0] : C.n_chunks;
    const int t_phys = C.dyn ? C.dyn[1] : C.t_phys;
    const int tid = (int)threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nw = kCullThreads / 32;
    if (tile * C.tile_size >= t_phys) {
        if (tid == 0) C.tile_items[tile] = 0;
        if (C.order) cull_last_orders(C);
        return;
    }
    // The boxes of the tile's warp segments (one segment: the whole tile),
    // one warp of this block per segment; the tile box is their union.
    const int seg_len = C.warp_targets > 0 ? C.warp_targets : C.tile_size;
    const int nseg = C.tile_size / seg_len;
    for (int sg = warp; sg < nseg; sg += nw) {
        int xl = 32767, yl = 32767, zl = 32767, xh = -32768, yh = -32768, zh = -32768;
        const int p0 = tile * C.tile_size + sg * seg_len;
        const int p1 = min(p0 + seg_len, t_phys);
        for (int p = p0 + lane; p < p1; p += 32) {
            const float4 t = C.tgt[p];
            if (t.w >= 0.f) {
                const int x = (int)t.x, y = (int)t.y, z = (int)t.z;
                xl = min(xl, x); yl = min(yl, y); zl = min(zl, z);
                xh = max(xh, x); yh = max(yh, y); zh = max(zh, z);
            }
        }
        warp_box(xl, yl, zl, xh, yh, zh);
        if (lane == 0) s_seg[sg] = make_box(xl, yl, zl, xh, yh, zh);
    }
    if (tid < kMaxItemsPerTile) s_cost[tid] = 0;
    if (C.hist)
        for (int w = tid; w < kMaxItemsPerTile * kMaxSegments; w += kCullThreads) s_wcost[w] = 0;
    __syncthreads();
    Box tb = s_seg[0];
    for (int sg = 1; sg < nseg; ++sg) {
        tb.xl = min(tb.xl, s_seg[sg].xl); tb.yl = min(tb.yl, s_seg[sg].yl);
        tb.zl = min(tb.zl, s_seg[sg].zl); tb.xh = max(tb.xh, s_seg[sg].xh);
        tb.yh = max(tb.yh, s_seg[sg].yh); tb.zh = max(tb.zh, s_seg[sg].zh);
    }
    int32_t* live = C.live + (size_t)tile * C.live_stride;
    int L = 0;
    for (int c0 = 0; c0 < n_chunks; c0 += kCullThreads) {
        const int c = c0 + tid;
        const bool on = c < n_chunks && box_gap2(tb, C.cbox[c]) < C.c2;
        const unsigned m = __ballot_sync(0xffffffffu, on);
        __syncthreads();  // s_wcount of the previous round is read
        if (lane == 0) s_wcount[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < nw; ++w) {
            before += w < warp ? s_wcount[w] : 0;
            total += s_wcount[w];
        }
        if (on) {
            const int li = L + before + __popc(m & ((1u << lane) - 1u));
            live[li] = c;
            if (li < kLiveSmem) s_live[li] = c;
        }
        L += total;
    }
    const int per = max(C.per_item, (L + C.max_items - 1) / C.max_items);
    const int nit = L == 0 ? 0 : (L + per - 1) / per;
    if (tid == 0) {  // the tile's first item: the claim's round trip overlaps the costs
        const int base = nit ? atomicAdd(C.item_count, nit) : 0;
        C.tile_first[tile] = base;
        C.tile_items[tile] = nit;
        s_base = base;
    }
    __syncthreads();  // the last round's live entries are visible to the block
    if (C.hist) {
        // item cost: the groups within the cutoff of each warp segment, one
        // thread per (live chunk, group), four group boxes in flight.  A CTA
        // takes an item as long as its busiest warp does: cost 4 x the most
        // groups of one segment + their mean over the segments.
        const int nw = L * kGroupsPerChunk;
        for (int w0 = tid; w0 < nw; w0 += 4 * kCullThreads) {
            Box gb[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * kCullThreads;
                if (w < nw) {
                    const int li = w / kGroupsPerChunk;
                    const int ch = L <= kLiveSmem ? s_live[li] : live[li];
                    gb[u] = C.gbox[(size_t)ch * kGroupsPerChunk + (w - li * kGroupsPerChunk)];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * kCullThreads;
                if (w < nw) {
                    const int it = (w / kGroupsPerChunk) / per;
                    for (int sg = 0; sg < nseg; ++sg)
                        if (box_gap2(s_seg[sg], gb[u]) < C.c2) atomicAdd(&s_wcost[it * nseg + sg], 1);
                }
            }
        }
        __syncthreads();
        for (int i = tid; i < nit; i += kCullThreads) {
            int mx = 0, sum = 0;
            for (int sg = 0; sg < nseg; ++sg) {
                mx = max(mx, s_wcost[i * nseg + sg]);
                sum += s_wcost[i * nseg + sg];
            }
            s_cost[i] = 4 * mx + sum / nseg;
        }
    }
    __syncthreads();
    for (int i = tid; i < nit; i += kCullThreads) {
        C.items[s_base + i] = make_int4(tile, i * per, min(per, L - i * per), s_cost[i]);
        if (C.hist) atomicAdd(&C.hist[min(s_cost[i], kCostBuckets - 1)], 1);
    }
    if (C.order) cull_last_orders(C);
}

// The pair sum over the work items (see the file comment).  KIND 0 point, 1
// gauss; PATH 0 MUFU rsqrt with the per-source warp vote, 1 the shared-memory
// table of w(k), 2 the shared-memory FP64 table of w(k) (1/sqrt(k) or the
// Gaussian term, whatever KIND) with the warp vote, every term added in FP64;
// NT threads, RP target pairs per thread (a warp owns 64 RP consecutive
// targets), SUB sources per FP32 run (SUB divides kGroup).  Partials go to
// A.part[item * tile_size + local target] (and A.part_norm).  Launched with a
// persistent grid and dynamic shared memory pair_smem_bytes(tab_k)
// (pair_smem_bytes64 for PATH 2).
//
// The items come from a problem set PS: one problem (a call of the API, one
// replica), or the culled replicas of a batch, whose items are numbered one
// after the other (ProblemList).  PS::count() is the number of items,
// PS::resolve(g, prob, local) the problem and local item of item g,
// PS::A(prob) / PS::C(prob) that problem's arguments, and PS::first() the
// arguments whose tables go to shared memory.
struct OneProblem {
    const PairArgs& a;
    const CullArgs& c;
    __device__ __forceinline__ int count() const { return *c.item_count; }
    __device__ __forceinline__ void resolve(int g, int& prob, int& local) const {
        prob = 0;
        local = c.order ? c.order[g] : g;
    }
    // the record of item g (in taking order) and its problem and local index
    __device__ __forceinline__ int4 item(int g, int& prob, int& local) const {
        prob = 0;
        if (c.oitems) {
            const int4 r = c.oitems[g];
            local = r.w;
            return r;
        }
        local = c.order ? c.order[g] : g;
        return c.items[local];
    }
    __device__ __forceinline__ const PairArgs& A(int) const { return a; }
    __device__ __forceinline__ const CullArgs& C(int) const { return c; }
    __device__ __forceinline__ const PairArgs& first() const { return a; }
    __device__ __forceinline__ int* work() const { return c.work; }
};
// The culled replicas list[0 .. n-1] of a batch, their arguments pa[r] and
// ca[r], and offs[i] the number of items of list[0 .. i-1] (offs[n] = all).
struct ProblemList {
    const PairArgs* pa;
    const CullArgs* ca;
    const int* list;
    const int* offs;   // [n + 2]: offs[n + 1] is the next item to take (zeroed with offs)
    int n;
    const int* order;  // the items largest first (null: in number order)
    __device__ __forceinline__ int count() const { return n > 0 ? offs[n] : 0; }
    __device__ __forceinline__ void resolve(int g, int& prob, int& local) const {
        if (order) g = order[g];
        int lo = 0, hi = n;  // the last i with offs[i] <= g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (offs[mid] <= g) lo = mid;
            else hi = mid;
        }
        prob = list[lo];
        local = g - offs[lo];
    }
    __device__ __forceinline__ int4 item(int g, int& prob, int& local) const {
        resolve(g, prob, local);
        return ca[prob].items[local];
    }
    __device__ __forceinline__ const PairArgs& A(int p) const { return pa[p]; }
    __device__ __forceinline__ const CullArgs& C(int p) const { return ca[p]; }
    __device__ __forceinline__ const PairArgs& first() const { return pa[list[0]]; }
    __device__ __forceinline__ int* work() const { return const_cast<int*>(offs) + n + 1; }
};

// The pairs of one staged chunk for one warp: the sources of its live groups
// (bit g of gmask: group g), in FP32 runs of SUB sources folded into acc64
// (PATH 0, 1), or term by term in FP64 (PATH 2).  sg/sq: the stage's source
// records; tx..tt: the warp's target pairs; nrm: the runs' |sums| (NORM).
//
// PIPE (PATH 0): the next source's r^2 is computed before the vote on this
// one, so that two independent chains are in flight across the branch; the
// arithmetic and the order of the additions are the same, and so are the bits.
// VOTE (PATH 0, without PIPE): sources per warp vote.  1: every source; 2 or
// 4: the r^2 of that many sources side by side, one vote on all of them;
// 0: no vote (the live group's every pair takes the rsqrt and the predicated
// FFMA).  A source that its vote lets through adds nothing unless a pair is
// inside the cutoff, and the additions keep the source order, so every VOTE
// gives the same bits.
template <int KIND, int PATH, int RP, int SUB, bool NORM, bool PIPE = false, int VOTE = 1>
__device__ __forceinline__ void chunk_pairs(const float4* __restrict__ sg,
                                            const float2* __restrict__ sq, const unsigned gmask,
                                            const float2 (&tx)[RP], const float2 (&ty)[RP],
                                            const float2 (&tz)[RP], const float2 (&tt)[RP],
                                            double (&acc64)[2 * RP],
                                            float (&nrm)[NORM ? 2 * RP : 1], const unsigned ulim,
                                            const int tab_k, const float* s_tab,
                                            const double* s_tab64) {
    const float2 half2 = f2(0.5f, 0.5f);
#pragma unroll 1
    for (int j0 = 0; j0 < CH; j0 += SUB) {
        if (!((gmask >> (j0 / kGroup)) & 1u)) continue;  // warp-uniform
        float acc[2 * RP];
#pragma unroll
        for (int k = 0; k < 2 * RP; ++k) acc[k] = 0.f;
        if constexpr (PATH == 0 && PIPE) {
            // r^2 - 1/2 of source j (three exact steps, as below)
            auto r2_of = [&](const int j, float2 (&u)[RP]) {
                const float4 g0 = sg[2 * j];
                const float4 g1 = sg[2 * j + 1];
                const float2 av = f2(g0.x, g0.y), bv = f2(g0.z, g0.w);
                const float2 cv = f2(g1.x, g1.y), dv = f2(g1.z, g1.w);
#pragma unroll
                for (int k = 0; k < RP; ++k) {
                    const float2 pa = __ffma2_rn(tx[k], av, tt[k]);
                    const float2 pc = __ffma2_rn(tz[k], cv, dv);
                    u[k] = __fadd2_rn(__ffma2_rn(ty[k], bv, pa), pc);
                }
            };
            float2 un[RP];
            r2_of(j0, un);
#pragma unroll 4
            for (int jj = 0; jj < SUB; ++jj) {
                float2 uu[RP];
                unsigned mk[RP];
#pragma unroll
                for (int k = 0; k < RP; ++k) {
                    uu[k] = un[k];
                    mk[k] = min(__float_as_uint(uu[k].x), __float_as_uint(uu[k].y));
                }
                // the next source (clamped inside the stage; unused past the run)
                r2_of(min(j0 + jj + 1, CH - 1), un);
#pragma unroll
                for (int w = 1; w < RP; w *= 2)
#pragma unroll
                    for (int k = 0; k + w < RP; k += 2 * w) mk[k] = min(mk[k], mk[k + w]);
                if (__any_sync(0xffffffffu, mk[0] < ulim)) {
                    const float qs = sq[j0 + jj].x;
#pragma unroll
                    for (int k = 0; k < RP; ++k) {
                        const float2 r2 = __fadd2_rn(uu[k], half2);
                        float wx = rsqrt_mufu(r2.x);
                        float wy = rsqrt_mufu(r2.y);
                        if (KIND == 1) {
                            const int ix =
                                min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, tab_k);
                            const int iy =
                                min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, tab_k);
                            wx = fminf(s_tab[ix], wx);
                            wy = fminf(s_tab[iy], wy);
                        }
                        fma_if_below(acc[2 * k], qs, wx, __float_as_uint(uu[k].x), ulim);
                        fma_if_below(acc[2 * k + 1], qs, wy, __float_as_uint(uu[k].y),
                                     ulim);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) acc64[k] += (double)acc[k];
            if (NORM) {
#pragma unroll
                for (int k = 0; k < 2 * RP; ++k) nrm[NORM ? k : 0] += fabsf(acc[k]);
            }
            continue;
        }
        if constexpr (PATH == 0 && VOTE != 1) {
            constexpr int V = VOTE == 0 ? 2 : VOTE;  // sources side by side
            static_assert(SUB % V == 0, "a vote's sources lie inside one FP32 run");
#pragma unroll(4 / V > 0 ? 4 / V : 1)
            for (int jj = 0; jj < SUB; jj += V) {
                float2 uu[V][RP];
                unsigned mk = 0xffffffffu;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = j0 + jj + v;
                    const float4 g0 = sg[2 * j];
                    const float4 g1 = sg[2 * j + 1];
                    const float2 av = f2(g0.x, g0.y), bv = f2(g0.z, g0.w);
                    const float2 cv = f2(g1.x, g1.y), dv = f2(g1.z, g1.w);
#pragma unroll
                    for (int k = 0; k < RP; ++k) {
                        const float2 pa = __ffma2_rn(tx[k], av, tt[k]);
                        const float2 pc = __ffma2_rn(tz[k], cv, dv);
                        uu[v][k] = __fadd2_rn(__ffma2_rn(ty[k], bv, pa), pc);
                        if (VOTE)
                            mk = min(mk, min(__float_as_uint(uu[v][k].x),
                                             __float_as_uint(uu[v][k].y)));
                    }
                }
                if (VOTE == 0 || __any_sync(0xffffffffu, mk < ulim)) {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        const float qs = sq[j0 + jj + v].x;
#pragma unroll
                        for (int k = 0; k < RP; ++k) {
                            const float2 r2 = __fadd2_rn(uu[v][k], half2);
                            float wx = rsqrt_mufu(r2.x);
                            float wy = rsqrt_mufu(r2.y);
                            if (KIND == 1) {
                                const int ix =
                                    min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, tab_k);
                                const int iy =
                                    min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, tab_k);
                                wx = fminf(s_tab[ix], wx);
                                wy = fminf(s_tab[iy], wy);
                            }
                            fma_if_below(acc[2 * k], qs, wx, __float_as_uint(uu[v][k].x), ulim);
                            fma_if_below(acc[2 * k + 1], qs, wy, __float_as_uint(uu[v][k].y),
                                         ulim);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) acc64[k] += (double)acc[k];
            if (NORM) {
#pragma unroll
                for (int k = 0; k < 2 * RP; ++k) nrm[NORM ? k : 0] += fabsf(acc[k]);
            }
            continue;
        }
        constexpr int kUnrollJ = PATH != 1 ? 4 : SUB;
#pragma unroll kUnrollJ
        for (int jj = 0; jj < SUB; ++jj) {
            const int j = j0 + jj;
            const float4 g0 = sg[2 * j];
            const float4 g1 = sg[2 * j + 1];
            const float2 av = f2(g0.x, g0.y), bv = f2(g0.z, g0.w);
            const float2 cv = f2(g1.x, g1.y), dv = f2(g1.z, g1.w);
            if constexpr (PATH == 2) {
                // r^2 - 1/2 exactly, the warp vote, then w(r^2) from the
                // FP64 table: r^2 = u + 1/2 and r^2 + 2^23 are exact in
                // FP32 (r^2 < 2^22), and the latter holds r^2 in its low
                // 23 mantissa bits; entries 0 and past the cutoff are 0,
                // so the clamped index also applies the cutoff and the
                // r = 0 skip
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
                if (__any_sync(0xffffffffu, mk[0] < ulim)) {
                    const double qd = (double)sq[j].x;
                    const float2 two23 = f2(8388608.f, 8388608.f);
#pragma unroll
                    for (int k = 0; k < RP; ++k) {
                        const float2 m2 = __fadd2_rn(__fadd2_rn(uu[k], half2), two23);
                        const int ix = min(__float_as_int(m2.x) & 0x7fffff, tab_k);
                        const int iy = min(__float_as_int(m2.y) & 0x7fffff, tab_k);
                        acc64[2 * k] = fma(qd, s_tab64[ix], acc64[2 * k]);
                        acc64[2 * k + 1] = fma(qd, s_tab64[iy], acc64[2 * k + 1]);
                    }
                }
            } else if constexpr (PATH == 0) {
                // r^2 - 1/2 in three exact steps and the warp vote, as
                // the SKIP tile of lgm_pairs.cuh
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
                if (__any_sync(0xffffffffu, mk[0] < ulim)) {
                    const float qs = sq[j].x;
#pragma unroll
                    for (int k = 0; k < RP; ++k) {
                        const float2 r2 = __fadd2_rn(uu[k], half2);
                        float wx = rsqrt_mufu(r2.x);
                        float wy = rsqrt_mufu(r2.y);
                        if (KIND == 1) {
                            const int ix =
                                min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, tab_k);
                            const int iy =
                                min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, tab_k);
                            wx = fminf(s_tab[ix], wx);
                            wy = fminf(s_tab[iy], wy);
                        }
                        fma_if_below(acc[2 * k], qs, wx, __float_as_uint(uu[k].x), ulim);
                        fma_if_below(acc[2 * k + 1], qs, wy, __float_as_uint(uu[k].y),
                                     ulim);
                    }
                }
            } else {
                const float qs = sq[j].x;
#pragma unroll
                for (int k = 0; k < RP; ++k) {
                    float2 u = __fadd2_rn(dv, tt[k]);
                    u = __ffma2_rn(tx[k], av, u);
                    u = __ffma2_rn(ty[k], bv, u);
                    u = __ffma2_rn(tz[k], cv, u);  // r^2 - 1/2, exact
                    const float2 r2 = __fadd2_rn(u, half2);
                    // w(k) from the table; entries 0 and c^2 are 0
                    const int ix =
                        min(__float_as_int(r2.x + 8388608.f) & 0x7fffff, tab_k);
                    const int iy =
                        min(__float_as_int(r2.y + 8388608.f) & 0x7fffff, tab_k);
                    fma_if_below(acc[2 * k], qs, s_tab[ix], __float_as_uint(u.x), ulim);
                    fma_if_below(acc[2 * k + 1], qs, s_tab[iy], __float_as_uint(u.y),
                                 ulim);
                }
            }
        }
        if constexpr (PATH != 2) {  // PATH 2 adds every term in FP64 already
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) acc64[k] += (double)acc[k];
        }
        if (NORM) {
#pragma unroll
            for (int k = 0; k < 2 * RP; ++k) nrm[NORM ? k : 0] += fabsf(acc[k]);
        }
    }
}

template <int KIND, int PATH, int NT, int RP, int SUB, bool NORM, class PS>
__device__ __forceinline__ void pair_items_culled(const PS& P) {
    static_assert(kGroup % SUB == 0, "an FP32 run lies inside one group");
    static_assert(PATH != 2 || !NORM, "the FP64-table path carries no FP32 run norms");
    constexpr int TS = NT * 2 * RP;
    const int nit = P.count();
    if ((int)blockIdx.x >= nit) return;
    // the shared-memory tables are the first problem's (a problem set shares them)
    const PairArgs& A0 = P.first();
    extern __shared__ __align__(128) unsigned char smem[];
    float4* s_geo = reinterpret_cast<float4*>(smem);                               // [2][CH*2]
    float2* s_qq = reinterpret_cast<float2*>(smem + 2 * CH * 2 * sizeof(float4));  // [2][CH]
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem + 2 * pair_stage_bytes());
    float* s_tab = reinterpret_cast<float*>(smem + 2 * pair_stage_bytes() + 16);
    double* s_tab64 = reinterpret_cast<double*>(smem + 2 * pair_stage_bytes() + 16);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_mbar_init();
    }
    if (PATH == 2) {
        for (int k = tid; k <= A0.tab_k; k += NT) s_tab64[k] = A0.tab64[k];
    } else if (KIND == 1 || PATH == 1) {
        for (int k = tid; k <= A0.tab_k; k += NT) s_tab[k] = A0.tab[k];
    }
    __syncthreads();

    // Producer (thread 0): walks this CTA's chunk sequence -- the live chunks
    // of items blockIdx.x, blockIdx.x + G, ... -- two chunks ahead.  Its
    // cursor lives in shared memory, out of the other threads' registers.
    // item, position, tile, first, count, chunks issued, problem
    __shared__ int s_prod[7];
    __shared__ Box s_wbox[NT / 32];
    // each stage also holds its chunk's four group boxes, copied with it
    __shared__ Box s_gbox[2][kGroupsPerChunk];
    auto load_item = [&](int g) {  // the producer's cursor onto item g
        int prob, local;
        P.resolve(g, prob, local);
        const int4 r = P.C(prob).items[local];
        s_prod[2] = r.x; s_prod[3] = r.y; s_prod[4] = r.z; s_prod[6] = prob;
    };
    auto issue_next = [&]() {
        int* Q = s_prod;
        if (Q[0] >= nit) return;
        const PairArgs& Ap = P.A(Q[6]);
        const CullArgs& Cp = P.C(Q[6]);
        const int chunk = Cp.live[(size_t)Q[2] * Cp.live_stride + Q[3] + Q[1]];
        const int st = Q[5] & 1;
        mbar_arrive_expect_tx(&s_bar[st],
                              (uint32_t)(pair_stage_bytes() + kGroupsPerChunk * sizeof(Box)));
        bulk_g2s(s_geo + st * CH * 2, Ap.geo + (size_t)chunk * CH * 2,
                 (uint32_t)(CH * 2 * sizeof(float4)), &s_bar[st]);
        bulk_g2s(s_qq + st * CH, Ap.qq + (size_t)chunk * CH, (uint32_t)(CH * sizeof(float2)),
                 &s_bar[st]);
        bulk_g2s(&s_gbox[st][0], Cp.gbox + (size_t)chunk * kGroupsPerChunk,
                 (uint32_t)(kGroupsPerChunk * sizeof(Box)), &s_bar[st]);
        ++Q[5];
        if (++Q[1] == Q[4]) {
            Q[0] += (int)gridDim.x;
            Q[1] = 0;
            if (Q[0] < nit) load_item(Q[0]);
        }
    };
    if (tid == 0) {
        s_prod[0] = (int)blockIdx.x; s_prod[1] = 0; s_prod[5] = 0;
        load_item((int)blockIdx.x);
        issue_next();
        issue_next();
    }

    uint32_t consumed = 0;
    bool failed = false;

    for (int it = (int)blockIdx.x; it < nit; it += (int)gridDim.x) {
        int prob, local;
        P.resolve(it, prob, local);
        const PairArgs& A = P.A(prob);
        const CullArgs& C = P.C(prob);
        const int t_phys = A.dyn ? A.dyn[1] : A.t_phys;
        const unsigned ulim = __float_as_uint(A.c2 - 0.5f);
        const int4 rec = C.items[local];
        const int tile = rec.x, count = rec.z;
        const int base = tile * TS;
        auto target_of = [&](int k) { return base + warp * (64 * RP) + k * 32 + lane; };
        float2 tx[RP], ty[RP], tz[RP], tt[RP];
        int xl = 32767, yl = 32767, zl = 32767, xh = -32768, yh = -32768, zh = -32768;
#pragma unroll
        for (int k = 0; k < RP; ++k) {
            const int p0 = target_of(2 * k), p1 = target_of(2 * k + 1);
            const float4 a = p0 < t_phys ? A.tgt[p0] : make_float4(0.f, 0.f, 0.f, -1.f);
            const float4 b = p1 < t_phys ? A.tgt[p1] : make_float4(0.f, 0.f, 0.f, -1.f);
            tx[k] = f2(a.x, b.x); ty[k] = f2(a.y, b.y); tz[k] = f2(a.z, b.z); tt[k] = f2(a.w, b.w);
            if (a.w >= 0.f) {
                xl = min(xl, (int)a.x); yl = min(yl, (int)a.y); zl = min(zl, (int)a.z);
                xh = max(xh, (int)a.x); yh = max(yh, (int)a.y); zh = max(zh, (int)a.z);
            }
            if (b.w >= 0.f) {
                xl = min(xl, (int)b.x); yl = min(yl, (int)b.y); zl = min(zl, (int)b.z);
                xh = max(xh, (int)b.x); yh = max(yh, (int)b.y); zh = max(zh, (int)b.z);
            }
        }
        warp_box(xl, yl, zl, xh, yh, zh);
        if (lane == 0) s_wbox[warp] = make_box(xl, yl, zl, xh, yh, zh);
        __syncwarp();

        double acc64[2 * RP];
        float nrm[NORM ? 2 * RP : 1];
#pragma unroll
        for (int k = 0; k < 2 * RP; ++k) acc64[k] = 0.0;
#pragma unroll
        for (int k = 0; k < (NORM ? 2 * RP : 1); ++k) nrm[k] = 0.f;

        for (int c = 0; c < count; ++c) {
            const int st = (int)(consumed & 1u);
            const uint32_t parity = (consumed >> 1) & 1u;
            const bool mine = mbar_wait_bounded(&s_bar[st], parity, A.err);
            if (!__syncthreads_and(mine)) { failed = true; break; }
            bool gon = false;
            if (lane < kGroupsPerChunk) gon = box_gap2(s_wbox[warp], s_gbox[st][lane]) < C.c2;
            const unsigned gmask = __ballot_sync(0xffffffffu, gon);
            if (C.examined && lane == 0 && gmask)
                atomicAdd(C.examined, (unsigned long long)__popc(gmask) * kGroup * 64 * RP);
            chunk_pairs<KIND, PATH, RP, SUB, NORM>(s_geo + st * CH * 2, s_qq + st * CH, gmask, tx, ty,
                                                   tz, tt, acc64, nrm, ulim, A.tab_k, s_tab,
                                                   s_tab64);
            __syncthreads();  // every thread is done with stage st
            ++consumed;
            if (tid == 0) {
                fence_proxy_async_smem();
                issue_next();
            }
        }
        if (failed) break;
        double* out = A.part + (size_t)local * TS;
#pragma unroll
        for (int k = 0; k < 2 * RP; ++k) {
            const int p = target_of(k);
            if (p < t_phys) {
                out[p - base] = acc64[k];
                if (NORM) A.part_norm[(size_t)local * TS + (p - base)] = nrm[NORM ? k : 0];
            }
        }
    }

    if (failed && tid == 0) {
        // A stage never completed: wait (bounded) for the copies still in
        // flight, then leave without results; the host sees DEVERR_TIMEOUT.
        mbar_drain_stages(s_bar, consumed, (uint32_t)s_prod[5]);
    }
}

// Dynamic shared memory of the warp-specialised kernel: S stages of source
// records and group boxes, their item records and full/empty barriers, then
// the table (elem bytes per entry; tab_k = 0 and elem = 0: none).
__host__ __device__ constexpr size_t ws_stage_bytes() {
    return pair_stage_bytes() + kGroupsPerChunk * sizeof(Box) + sizeof(int4) + 2 * sizeof(uint64_t);
}
inline size_t ws_smem_bytes(int S, int tab_k, int elem) {
    return (size_t)S * ws_stage_bytes() + (size_t)(tab_k + 1) * elem + 16;
}

// The pair sum over the work items, warp-specialised.  NW consumer warps own
// the tile's targets as in pair_items_culled (TS = NW * 64 RP); one producer
// warp (its lane 0) takes items from an atomic counter -- whichever CTA is
// free takes the next item -- and streams their chunks through an S-stage
// ring: stage records {local item, chunk position, chunks, problem} and the
// item's tile, full barriers (the bulk copies) and empty barriers (one
// arrival per consumer warp).  The producer claims the next item only when
// the consumers are on the last chunk it issued (see the claim below).  Consumer warps never wait for one another: a warp whose groups are
// all beyond the cutoff of its targets passes a chunk at once, and may run up
// to S chunks ahead of the slowest warp.  After the last item the producer
// posts a record with item -1 (no copy) that ends the consumers.  Every wait
// is bounded: on a timeout the warp raises DEVERR_TIMEOUT and leaves, the
// producer's own waits then run out, and it waits (bounded) for the copies it
// has in flight before leaving.  Per target, chunks and FP32 runs are added
// in the order of pair_items_culled: the sums are bit for bit the same.
template <int KIND, int PATH, int NW, int RP, int SUB, bool NORM, int S, bool PIPE, class PS,
          int VOTE = 1>
__device__ __forceinline__ void pair_items_culled_ws(const PS& P) {
    static_assert(kGroup % SUB == 0, "an FP32 run lies inside one group");
    static_assert(PATH != 2 || !NORM, "the FP64-table path carries no FP32 run norms");
    constexpr int NT = NW * 32;
    constexpr int TS = NT * 2 * RP;
    const int nit = P.count();
    if ((int)blockIdx.x >= nit) return;
    const PairArgs& A0 = P.first();
    extern __shared__ __align__(128) unsigned char smem[];
    float4* s_geo = reinterpret_cast<float4*>(smem);                               // [S][CH*2]
    float2* s_qq = reinterpret_cast<float2*>(smem + S * CH * 2 * sizeof(float4));  // [S][CH]
    Box* s_gbox = reinterpret_cast<Box*>(smem + S * pair_stage_bytes());  // [S][groups]
    int4* s_rec = reinterpret_cast<int4*>(smem + S * (pair_stage_bytes() +
                                                      kGroupsPerChunk * sizeof(Box)));
    uint64_t* s_full = reinterpret_cast<uint64_t*>(s_rec + S);
    uint64_t* s_empty = s_full + S;
    float* s_tab = reinterpret_cast<float*>(smem + S * ws_stage_bytes());
    double* s_tab64 = reinterpret_cast<double*>(smem + S * ws_stage_bytes());
    __shared__ Box s_wbox[NW];
    __shared__ int s_tile[S];  // the tile of each stage's item

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(&s_full[i], 1);
            mbar_init(&s_empty[i], NW);
        }
        fence_mbar_init();
    }
    if (PATH == 2) {
        for (int k = tid; k <= A0.tab_k; k += NT + 32) s_tab64[k] = A0.tab64[k];
    } else if (KIND == 1 || PATH == 1) {
        for (int k = tid; k <= A0.tab_k; k += NT + 32) s_tab[k] = A0.tab[k];
    }
    __syncthreads();

    if (warp == NW) {  // the producer warp
        if (lane != 0) return;
        unsigned* err = A0.err;
        uint32_t k = 0;  // stages issued
        bool ok = true;
        for (;;) {
            // Claim the next item only once the target warps have released
            // every chunk but the last one issued.  Claimed but unstarted
            // items are what the other CTAs wait for at the end of the
            // kernel: taken early, the largest items would pile up three to
            // a CTA in the first microseconds.  The claim and the first copy
            // take less than a chunk's sums.
            if (k >= 2 && !mbar_wait_bounded(&s_empty[(k - 2) % S], ((k - 2) / S) & 1u, err)) {
                ok = false;
                break;
            }
            const int g = atomicAdd(P.work(), 1);
            const bool done = g >= nit;
            if (done) pdl_trigger();  // no item left: the next kernel may be scheduled
            int prob = 0, local = -1;
            int4 r = make_int4(0, 0, 1, 0);
            if (!done) r = P.item(g, prob, local);
            for (int c = 0; c < r.z; ++c, ++k) {
                const int st = (int)(k % S);
                if (k >= (uint32_t)S && !mbar_wait_bounded(&s_empty[st], (k / S - 1) & 1u, err)) {
                    ok = false;
                    break;
                }
                s_rec[st] = make_int4(local, c, r.z, prob);
                s_tile[st] = r.x;
                if (done) {
                    mbar_arrive(&s_full[st]);  // the end record: no copy
                } else {
                    const PairArgs& Ap = P.A(prob);
                    const CullArgs& Cp = P.C(prob);
                    const int chunk = Cp.live[(size_t)r.x * Cp.live_stride + r.y + c];
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(&s_full[st], (uint32_t)(pair_stage_bytes() +
                                                                  kGroupsPerChunk * sizeof(Box)));
                    bulk_g2s(s_geo + st * CH * 2, Ap.geo + (size_t)chunk * CH * 2,
                             (uint32_t)(CH * 2 * sizeof(float4)), &s_full[st]);
                    bulk_g2s(s_qq + st * CH, Ap.qq + (size_t)chunk * CH,
                             (uint32_t)(CH * sizeof(float2)), &s_full[st]);
                    bulk_g2s(s_gbox + st * kGroupsPerChunk,
                             Cp.gbox + (size_t)chunk * kGroupsPerChunk,
                             (uint32_t)(kGroupsPerChunk * sizeof(Box)), &s_full[st]);
                }
            }
            if (!ok || done) break;
        }
        // a consumer that gave up leaves copies unconsumed: let them land first
        if (!ok) mbar_drain_ring(s_full, S, k > (uint32_t)S ? k - S : 0u, k);
        return;
    }

    // consumer warps
    float2 tx[RP], ty[RP], tz[RP], tt[RP];
    double acc64[2 * RP];
    float nrm[NORM ? 2 * RP : 1];
    int base = 0, t_phys = 0, c2 = 0, tab_k = 0;
    unsigned ulim = 0;
    auto target_of = [&](int q) { return base + warp * (64 * RP) + q * 32 + lane; };
    for (uint32_t k = 0;; ++k) {
        const int st = (int)(k % S);
        // every lane waits (acquiring the copy), and the warp leaves as one
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_full[st], (k / S) & 1u, A0.err)))
            break;
        const int4 m = s_rec[st];
        if (m.x < 0) break;  // the end record
        const PairArgs& A = P.A(m.w);
        const CullArgs& C = P.C(m.w);
        if (m.y == 0) {  // the item's first chunk: its tile's targets of this warp
            base = s_tile[st] * TS;
            t_phys = A.dyn ? A.dyn[1] : A.t_phys;
            c2 = C.c2;
            tab_k = A.tab_k;
            ulim = __float_as_uint(A.c2 - 0.5f);
            int xl = 32767, yl = 32767, zl = 32767, xh = -32768, yh = -32768, zh = -32768;
#pragma unroll
            for (int q = 0; q < RP; ++q) {
                const int p0 = target_of(2 * q), p1 = target_of(2 * q + 1);
                const float4 a = p0 < t_phys ? A.tgt[p0] : make_float4(0.f, 0.f, 0.f, -1.f);
                const float4 b = p1 < t_phys ? A.tgt[p1] : make_float4(0.f, 0.f, 0.f, -1.f);
                tx[q] = f2(a.x, b.x); ty[q] = f2(a.y, b.y); tz[q] = f2(a.z, b.z);
                tt[q] = f2(a.w, b.w);
                if (a.w >= 0.f) {
                    xl = min(xl, (int)a.x); yl = min(yl, (int)a.y); zl = min(zl, (int)a.z);
                    xh = max(xh, (int)a.x); yh = max(yh, (int)a.y); zh = max(zh, (int)a.z);
                }
                if (b.w >= 0.f) {
                    xl = min(xl, (int)b.x); yl = min(yl, (int)b.y); zl = min(zl, (int)b.z);
                    xh = max(xh, (int)b.x); yh = max(yh, (int)b.y); zh = max(zh, (int)b.z);
                }
            }
            warp_box(xl, yl, zl, xh, yh, zh);
            if (lane == 0) s_wbox[warp] = make_box(xl, yl, zl, xh, yh, zh);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 2 * RP; ++q) acc64[q] = 0.0;
#pragma unroll
            for (int q = 0; q < (NORM ? 2 * RP : 1); ++q) nrm[q] = 0.f;
        }
        bool gon = false;
        if (lane < kGroupsPerChunk)
            gon = box_gap2(s_wbox[warp], s_gbox[st * kGroupsPerChunk + lane]) < c2;
        const unsigned gmask = __ballot_sync(0xffffffffu, gon);
        if (C.examined && lane == 0 && gmask)
            atomicAdd(C.examined, (unsigned long long)__popc(gmask) * kGroup * 64 * RP);
        chunk_pairs<KIND, PATH, RP, SUB, NORM, PIPE, VOTE>(s_geo + st * CH * 2, s_qq + st * CH,
                                                           gmask, tx, ty, tz, tt, acc64, nrm,
                                                           ulim, tab_k, s_tab, s_tab64);
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_empty[st]);  // this warp is done with stage st
        if (m.y == m.z - 1) {  // the item's last chunk: its partials
            double* out = A.part + (size_t)m.x * TS;
#pragma unroll
            for (int q = 0; q < 2 * RP; ++q) {
                const int p = target_of(q);
                if (p < t_phys) {
                    out[p - base] = acc64[q];
                    if (NORM) A.part_norm[(size_t)m.x * TS + (p - base)] = nrm[NORM ? q : 0];
                }
            }
        }
    }
}

template <int KIND, int PATH, int NT, int RP, int SUB, bool NORM = false>
__global__ void __launch_bounds__(NT) pair_kernel_culled(PairArgs A, CullArgs C) {
    pdl_wait();
    pdl_trigger();
    pair_items_culled<KIND, PATH, NT, RP, SUB, NORM>(OneProblem{A, C});
}

// The culled replicas of a batch in one persistent launch (point charges,
// MUFU path): their items are numbered one after the other (ProblemList).
template <int NT, int RP, int SUB, bool NORM>
__global__ void __launch_bounds__(NT) pair_kernel_culled_list(ProblemList L) {
    pair_items_culled<0, 0, NT, RP, SUB, NORM>(L);
}

// Warp-specialised: NW consumer warps and one producer warp, S stages, at
// least MINB resident CTAs per SM (a register bound).
template <int KIND, int PATH, int NW, int RP, int SUB, int S, int MINB, bool NORM = false,
          bool PIPE = false, int VOTE = 1>
__global__ void __launch_bounds__(NW * 32 + 32, MINB)
    pair_kernel_culled_ws(PairArgs A, CullArgs C) {
    pdl_wait();
    pair_items_culled_ws<KIND, PATH, NW, RP, SUB, NORM, S, PIPE, OneProblem, VOTE>(
        OneProblem{A, C});
}
template <int NW, int RP, int SUB, int S, int MINB, bool NORM, bool PIPE = false, int VOTE = 1>
__global__ void __launch_bounds__(NW * 32 + 32, MINB) pair_kernel_culled_ws_list(ProblemList L) {
    pair_items_culled_ws<0, 0, NW, RP, SUB, NORM, S, PIPE, ProblemList, VOTE>(L);
}

// (static: each translation unit that launches them has its own copy)
static __global__ void __launch_bounds__(CH) chunk_boxes_kernel(PairArgs A, CullArgs C) {
    pdl_wait();
    pdl_trigger();
    chunk_boxes_body(A, C, (int)blockIdx.x);
}

static __global__ void __launch_bounds__(kCullThreads) cull_kernel(CullArgs C) {
    pdl_wait();
    pdl_trigger();
    cull_body(C, (int)blockIdx.x);
}

static __global__ void __launch_bounds__(1024) order_items_kernel(CullArgs C) {
    order_items_body(C);
}

// Sum of one physical target's item partials (its tile's items, in order).
__device__ __forceinline__ double item_sum(const double* __restrict__ part,
                                           const int* __restrict__ tile_first,
                                           const int* __restrict__ tile_items, int tile_size,
                                           int p) {
    const int tile = p / tile_size, loc = p - tile * tile_size;
    const int n = tile_items[tile];
    const double* q = part + (size_t)tile_first[tile] * tile_size + loc;
    double s = 0.0;
    int i = 0;
    for (; i + 4 <= n; i += 4) {  // four loads in flight, then the adds in order
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = q[(size_t)(i + u) * tile_size];
#pragma unroll
        for (int u = 0; u < 4; ++u) s += v[u];
    }
    for (; i < n; ++i) s += q[(size_t)i * tile_size];
    return s;
}

}  // namespace lgm
