// lgm_context.hpp -- host-side state behind an lgm_ctx handle.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "langmuir_b200.h"

struct lgm_ctx {
    lgm_config cfg{};
    int device = 0;
    int sm_count = 0;
    int volume = 0;
    int xy = 0;
    cudaStream_t stream = nullptr;

    // Device work buffers, grown on demand (never inside stream capture).
    float4* d_geo = nullptr;  size_t geo_cap = 0;   // 2 float4 per source
    float2* d_qq = nullptr;   size_t qq_cap = 0;    // 1 float2 per source
    float4* d_tgt = nullptr;  size_t tgt_cap = 0;   // per physical target
    double* d_part = nullptr; size_t part_cap = 0;  // split partial sums
    int32_t* d_s = nullptr;   size_t s_cap = 0;     // staging for host-buffer calls
    int32_t* d_q = nullptr;   size_t q_cap = 0;
    int32_t* d_t = nullptr;   size_t t_cap = 0;
    double* d_o = nullptr;    size_t o_cap = 0;
    float* d_gtab = nullptr;  int gtab_k = 0;       // gauss correction table
    float* d_rtab = nullptr;  int rtab_k = 0;       // 1/sqrt(k) table
    double* d_rtab64 = nullptr;                      // FP64 1/sqrt(k) (TABLE64 path)
    double* d_gtab64 = nullptr;                      // FP64 erf(f sqrt(k))/sqrt(k) (TABLE64)
    unsigned* d_err = nullptr;                       // device error word

    // Spatial order of the targets: a target's bin is the Morton rank of its
    // lattice cell (cubes of 2^cell_shift sites); a counting sort by bin gives
    // the permutation the pair tiles run in (perm[physical] = target).
    int cell_shift = 2, cells_x = 0, cells_y = 0, ncells = 0;
    int32_t* d_cell_rank = nullptr;                  // [ncells]
    int32_t* d_bins = nullptr;                       // [ncells + 2] counts, then offsets
    int32_t* d_key = nullptr;  size_t key_cap = 0;   // bin per target
    int32_t* d_perm = nullptr; size_t perm_cap = 0;  // target of each physical slot
    int32_t* d_ttmp = nullptr; size_t ttmp_cap = 0;  // targets scattered by bin
    // The sources in the same spatial order: bin per source (d_sbins follows
    // the target bins in the d_bins allocation), the sources scattered by bin,
    // then ranked inside their bin by (site, index), so that the order is a
    // function of the sources alone.
    int32_t* d_sbins = nullptr;                       // [ncells + 2], inside d_bins
    int bins_stride = 0;                              // ncells + 2 rounded up to 4
    int32_t* d_skey = nullptr; size_t skey_cap = 0;   // bin per source
    int32_t* d_stmp = nullptr; size_t stmp_cap = 0;   // sources scattered by bin
    // Culled pair sums (lgm_cull.cuh): chunk and group boxes, live chunk
    // lists per tile, work items, and where each tile's items start.
    int4* d_cbox = nullptr;  size_t cbox_cap = 0;     // lgm::Box per chunk
    int4* d_gbox = nullptr;  size_t gbox_cap = 0;     // lgm::Box per 32-source group
    int32_t* d_live = nullptr; size_t live_cap = 0;
    int4* d_items = nullptr; size_t items_cap = 0;
    int32_t* d_tile_first = nullptr; size_t tfirst_cap = 0;
    int32_t* d_tile_items = nullptr; size_t titems_cap = 0;
    int32_t* d_item_count = nullptr;                  // [3]: items written, next item taken,
                                                      // tiles culled
    int32_t* d_cost_hist = nullptr;                   // [kCostBuckets] items per cost
    int32_t* d_order = nullptr; size_t order_cap = 0; // items by decreasing cost
    int4* d_oitems = nullptr; size_t oitems_cap = 0;  // their records in that order

    // Pinned host staging for the host-buffer entry points.
    int32_t* h_s = nullptr;   size_t hs_cap = 0;
    int32_t* h_q = nullptr;   size_t hq_cap = 0;
    int32_t* h_t = nullptr;   size_t ht_cap = 0;
    double* h_o = nullptr;    size_t ho_cap = 0;
    unsigned* h_err = nullptr;

    int bps[40][4] = {};                 // resident CTAs per SM, per variant and kernel
    int forced_variant = -1;             // -1: autotuned / default
    std::map<uint64_t, int> tune_cache;  // size bucket -> fastest variant

    bool counting = false;
    unsigned long long* d_examined = nullptr;  // pairs examined by the last culled launch
    bool count_pending = false;
    bool timing = false;
    cudaEvent_t ev_pair0 = nullptr, ev_pair1 = nullptr;  // bracket the pair kernel
    // the call's kernels launched with programmatic stream serialization
    // (lgm_set_launch_overlap), and both bin arrays known to be zero (the
    // last kernel of a completed launch sequence clears them)
    bool overlap = true;
    bool bins_clean = false;
    bool timed_pending = false;

    std::string err;
    lgm_launch_info last{};
};
