// lgm_kmc.cu -- one Langmuir kMC replica stepped entirely on the GPU.
//
// Step (Simulation::performIterations, transistor set-up, simulation.cpp:34-111),
// as a chain of kernels that read every count from device memory, so one
// step is captured once as a CUDA graph and replayed:
//   choose     proposals, ChargeAgent::chooseFuture (chargeagent.cpp:73-78)
//   pack       source / target records for the Coulomb sums (kernel-2 layout)
//   pair       FP32 pair sums + per-target error scale N (lgm_pairs.cuh)
//   finalize   potentials V and N per target
//   decide     ChargeAgent::decideFuture (chargeagent.cpp:90-161): Metropolis
//              with coupling, drains; decisions whose energy lies within the
//              FP32 error bound of the acceptance threshold are queued
//   guard      those decisions redone with FP64 sums (the oracle's arithmetic)
//   claim/move completeTick in list order (chargeagent.cpp:163-199): the lowest
//              list index wins a contested site; drains remove the carrier
//   compact    Simulation::nextTick list removal + the four electrode sources'
//              tryToInject (sourceagent.cpp:92-103) + currentStep += 1
// Random numbers come from the counter-based stream of lgm_rng.cuh, the
// stream the oracle (oracle/lgm_oracle_kmc.cpp) uses, so occupancies and
// decisions compare bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "langmuir_b200_kmc.h"
#include "lgm_cull.cuh"
#include "lgm_rng.cuh"

using namespace lgm;

namespace {

// Agent::Type (include/agent.h:33-55) in the per-site type arrays.
enum : uint8_t { T_EMPTY = 0, T_ELECTRON = 1, T_HOLE = 2, T_DEFECT = 3, T_SOURCE = 4, T_DRAIN = 5 };
// Special agent ids above the lattice (Grid::registerSpecialAgent in the order
// of World::createSources/createDrains, world.cpp:961-1187).
constexpr int kSpecial = 35;
constexpr int E_DRAIN_L = 3, E_DRAIN_R = 4, H_DRAIN_L = 2, H_DRAIN_R = 3;
// Outcomes (same codes as the oracle).
enum : int32_t { O_OCCUPIED = 0, O_MET_ACCEPT = 1, O_MET_REJECT = 2, O_DRAIN_ACCEPT = 3,
                 O_DRAIN_REJECT = 4 };
// Device counters: 20 flux (attempts, successes) + proposals + accepted + guard.
enum { C_XSRC = 16, C_RECOMB = 18, C_PROPOSALS = 20, C_ACCEPTED = 21, C_GUARD = 22, C_NUM = 23 };
// Device ints.
// I_FIRST_E/H: the lowest list index a step removes (INT_MAX: none), where
// the stable compaction of that list starts.
enum { I_NE = 0, I_NH, I_STEP, I_NFLAG, I_REMOVED, I_NE0, I_NH0, I_NCHUNK, I_TPHYS, I_TPAD,
       I_NBONDS, I_FIRST_E, I_FIRST_H, I_NUM };
// Recombination, exciton-source and charge-balancing purposes of the random
// stream (balancing try t of electrons draws at {step, t, RNG_BALANCE_E}, its
// side at {step, t, RNG_BALANCE_E + 1}; holes at RNG_BALANCE_H, + 1).
constexpr uint32_t RNG_RECOMB = 5, RNG_EXCITON = RNG_SOURCE + 4;
constexpr uint32_t RNG_BALANCE_E = RNG_SOURCE + 8, RNG_BALANCE_H = RNG_SOURCE + 10;
// Tries of one species' balancing per step before the reference gives up
// (Simulation::balanceCharges, simulation.cpp:272-276).
constexpr int kBalanceTries = 1024;

// Guard band: FP32C potentials carry at most (2 ulp rsqrt + 31 u run sums)
// ~ 2.1e-6 N of error each; a decision whose energy lies within
// guard*(N_c + N_f) of the threshold is redone in FP64, with guard =
// lgm_params::guard_band >= LGM_GUARD_BAND_MIN (8e-6).

constexpr int kNT = 128, kRP = 4, kSUB = 32;
constexpr int kTile = kNT * 2 * kRP;
constexpr int kCullPerItem = 2;  // source chunks per work item of the culled pair sum
// The culled pair sum: the warp-specialised kernel (lgm_cull.cuh) with 4
// target warps of 2 target pairs per thread, a producer warp, 4 stages and 4
// resident CTAs per SM; items taken largest first (the API's default variant).
constexpr int kCNW = 4, kCRP = 2, kCStages = 4, kCMinBlocks = 4;
constexpr int kCSUB = kGroup;  // FP32 runs of the culled sum: one source group
constexpr int kCVote = 2;      // sources per warp vote of the culled sum (the same bits)
constexpr int kCThreads = kCNW * 32 + 32;
constexpr int kCTile = kCNW * 32 * 2 * kCRP;
// Replicas with room for fewer source chunks than this keep the unculled
// skip tile: with a handful of chunks the boxes and the cull only add launches.
constexpr int kCullMinChunks = 8;

struct Dev {
    int X, Y, Z, XY, V, hr;
    int cap_e, cap_h, nd, dq;
    uint32_t seed, replica;
    double beta, exciton_binding, sI100, prefactor, erffactor;
    double guard;  // guard band width relative to N (lgm_params::guard_band)
    double coupling[27];
    double rate_src[4], rate_drain[4];  // eL eR hL hR
    int coulomb, gauss;
    unsigned terms;  // LGM_TERM_* bits
    int nterms;
    int cutoff2;
    double* pot;
    uint8_t *et, *ht;
    int32_t *e_site, *h_site, *e_f, *h_f, *defects;
    int32_t *claim_e, *claim_h;
    int32_t* outcome;
    double* de;
    uint8_t* accept;
    int32_t* flagged;
    // the guard's per-split FP64 partials [ncap][kGuardSplits] and, per queued
    // decision, the splits done (the last one sums them; zero between steps)
    double2* gpart;
    int32_t* gdone;
    int32_t* cnt;
    unsigned long long* ctr;
    float4* geo;
    float2* qq;
    float4* tgt;
    double* part;
    float* part_norm;
    double *Vt, *Nt;
    double* w64;          // FP64 w(k) for integer r^2 = k < cutoff^2 (w(0) = 0), the guard's table
    const float* gtab;    // Gaussian charges: the pair kernel's FP32 erf(f r)/r table
    int gtab_k;           // its last index (NaN there: past it the term is 1/r)
    // Targets in lattice-cell order for the skip pair tiles (sorted != 0): a
    // counting sort by the Morton rank of each target's cell; tperm[slot] is
    // the target in physical slot `slot`.
    int sorted, cell_shift, cells_x, cells_y, ncells;
    const int32_t* cell_rank;  // [ncells]
    int32_t* bins;             // [ncells + 2]
    int32_t *tkey, *tperm;     // [2 ncap]
    int splits;
    // Culled pair sums (lgm_cull.cuh; standalone replicas and a batch's
    // per-phase replicas of point charges): the sources sorted by (charge
    // class, lattice cell) and by site inside a bin (skey: bin per source,
    // stmp: sources scattered by bin, sbins: 3 (ncells + 1) bin counters), the
    // targets scattered by bin before their rank inside it (ttmp, [2 ncap]),
    // chunk and group boxes, each tile's live chunks and the work items.  A
    // charge class stays padded to whole chunks.
    int culled, max_items;
    int32_t *skey, *stmp, *sbins, *ttmp;
    Box *cbox, *gbox;
    int32_t* live;
    int4* items;
    int32_t *item_count, *tile_first, *tile_items;  // item_count[3]: written, taken, tiles
                                                    // culled
    int32_t *chist, *corder;  // item costs' histogram and the largest-first order
                              // (corder null for a batch's replicas: the batch's)
    int src_cap;   // source records capacity (multiple of CH)
    int tpad_cap;  // per-term target block capacity
    unsigned* err;
    // injection energetics (sourceagent.cpp:125-181) and charge balancing
    // (simulation.cpp:253-353): source.metropolis, source.coulomb,
    // balance.charges, and the electrode voltages that pick the balancing side
    int src_metro, src_coulomb, balance;
    double volt_l, volt_r;
    // solar-cell set-up
    int solar, rec_range, confine, gen_iface;
    double gen_rate, rec_rate;
    uint8_t* phase;       // donor 0 / acceptor 1 per site (extensions)
    int32_t* bonds;       // donor, acceptor site pairs
    int32_t* h_at;        // hole index at a site, -1 elsewhere (recombination)
    int32_t* rclaim;      // per hole: lowest successful recombining electron
    int32_t* e_rch;       // per electron: chosen hole, -1 if none
    uint8_t *e_rm, *h_rm; // removed by recombination this step
};

// ---- lattice helpers (cubicgrid.cpp:132-165, 207-471) ---------------------------
__device__ __forceinline__ void xyz(const Dev& D, int s, int& x, int& y, int& z) {
    z = s / D.XY;
    y = s / D.X - z * D.Y;
    x = s % D.X;
}
__device__ __forceinline__ int sidx(const Dev& D, int x, int y, int z) {
    return D.X * (y + z * D.Y) + x;
}

// Grid::neighborsSite in the reference's push order, then the face drains.
__device__ int neighbors(const Dev& D, int site, bool electron, int* nb, int range) {
    int x, y, z;
    xyz(D, site, x, y, z);
    const int X = D.X, Y = D.Y, Z = D.Z;
    int n = 0;
    auto S = [&](int a, int b, int c) { nb[n++] = sidx(D, a, b, c); };
    if (range == 1) {
        if (x > 0) S(x - 1, y, z);
        if (x < X - 1) S(x + 1, y, z);
        if (y > 0) S(x, y - 1, z);
        if (y < Y - 1) S(x, y + 1, z);
        if (z > 0) S(x, y, z - 1);
        if (z < Z - 1) S(x, y, z + 1);
    } else if (Z == 1) {
        if (x > 0) { S(x - 1, y, z); if (y > 0) S(x - 1, y - 1, z); if (y < Y - 1) S(x - 1, y + 1, z); if (x > 1) S(x - 2, y, z); }
        if (x < X - 1) { S(x + 1, y, z); if (y > 0) S(x + 1, y - 1, z); if (y < Y - 1) S(x + 1, y + 1, z); if (x < X - 2) S(x + 2, y, z); }
        if (y > 0) { S(x, y - 1, z); if (y > 1) S(x, y - 2, z); }
        if (y < Y - 1) { S(x, y + 1, z); if (y < Y - 2) S(x, y + 2, z); }
    } else {
        if (x > 0) {
            S(x - 1, y, z);
            if (y > 0) { S(x - 1, y - 1, z); if (z > 0) S(x - 1, y - 1, z - 1); if (z < Z - 1) S(x - 1, y - 1, z + 1); }
            if (y < Y - 1) { S(x - 1, y + 1, z); if (z > 0) S(x - 1, y + 1, z - 1); if (z < Z - 1) S(x - 1, y + 1, z + 1); }
            if (z > 0) S(x - 1, y, z - 1);
            if (z < Z - 1) S(x - 1, y, z + 1);
            if (x > 1) S(x - 2, y, z);
        }
        if (x < X - 1) {
            S(x + 1, y, z);
            if (y > 0) { S(x + 1, y - 1, z); if (z > 0) S(x + 1, y - 1, z - 1); if (z < Z - 1) S(x + 1, y - 1, z + 1); }
            if (y < Y - 1) { S(x + 1, y + 1, z); if (z > 0) S(x + 1, y + 1, z - 1); if (z < Z - 1) S(x + 1, y + 1, z + 1); }
            if (z > 0) S(x + 1, y, z - 1);
            if (z < Z - 1) S(x + 1, y, z + 1);
            if (x < X - 2) S(x + 2, y, z);
        }
        if (z > 0) { S(x, y, z - 1); if (y > 0) S(x, y - 1, z - 1); if (y < Y - 1) S(x, y + 1, z - 1); if (z > 1) S(x, y, z - 2); }
        if (z < Z - 1) { S(x, y, z + 1); if (y > 0) S(x, y - 1, z + 1); if (y < Y - 1) S(x, y + 1, z + 1); if (z < Z - 2) S(x, y, z + 2); }
        if (y > 0) { S(x, y - 1, z); if (y > 1) S(x, y - 2, z); }
        if (y < Y - 1) { S(x, y + 1, z); if (y < Y - 2) S(x, y + 2, z); }
    }
    if (x == 0) nb[n++] = D.V + (electron ? E_DRAIN_L : H_DRAIN_L);
    if (x == X - 1) nb[n++] = D.V + (electron ? E_DRAIN_R : H_DRAIN_R);
    return n;
}

__device__ __forceinline__ Philox4 draw(const Dev& D, uint32_t step, uint32_t index,
                                        uint32_t purpose) {
    return philox4x32_10(step, index, purpose, 0u, D.seed, D.replica);
}

// ---- kernels ----------------------------------------------------------------------

// Proposals; also snapshots the step's carrier counts.
__device__ __forceinline__ void choose_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    const uint32_t step = (uint32_t)D.cnt[I_STEP];
    if (i == 0) {
        D.cnt[I_NE0] = ne;
        D.cnt[I_NH0] = nh;
        D.cnt[I_NFLAG] = 0;
        D.cnt[I_REMOVED] = 0;
        D.cnt[I_FIRST_E] = INT_MAX;
        D.cnt[I_FIRST_H] = INT_MAX;
    }
    if (i >= ne + nh) return;
    const bool e = i < ne;
    const int k = e ? i : i - ne;
    (e ? D.e_rm : D.h_rm)[k] = 0;
    const int site = e ? D.e_site[k] : D.h_site[k];
    int nb[40];
    const int n = neighbors(D, site, e, nb, D.hr);
    const Philox4 r = draw(D, step, (uint32_t)k, e ? RNG_CHOOSE_E : RNG_CHOOSE_H);
    const int f = nb[uint_below(r.w[0], (uint32_t)n)];
    (e ? D.e_f : D.h_f)[k] = f;
}

// Site of source i in list order: electrons, holes, then defects.
__device__ __forceinline__ int src_site(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    if (i < ne) return D.e_site[i];
    if (i < ne + nh) return D.h_site[i - ne];
    return D.defects[i - ne - nh];
}

// Source records (electrons, holes, defects, each padded to whole chunks so
// that every FP32 run holds one charge sign) and target records (current sites
// then future sites, one block per term).
__device__ __forceinline__ void pack_body(const Dev& D, const int j) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    const int nd = D.dq != 0 ? D.nd : 0;
    const int pe = (ne + CH - 1) / CH * CH, ph = (nh + CH - 1) / CH * CH,
              pd = (nd + CH - 1) / CH * CH;
    const int nsrc = pe + ph + pd;
    const int t = 2 * (ne + nh);
    const int tpad = (t + 63) / 64 * 64;
    if (j == 0) {
        D.cnt[I_NCHUNK] = nsrc / CH;
        D.cnt[I_TPHYS] = D.nterms * tpad;
        D.cnt[I_TPAD] = tpad;
    }
    auto record = [&](int dst, int s, float q) {
        float a = 0.f, b = 0.f, c = 0.f, d = -0.5f;
        if (s >= 0) {
            int x, y, z;
            xyz(D, s, x, y, z);
            a = -2.f * x; b = -2.f * y; c = -2.f * z;
            d = (float)(x * x + y * y + z * z) - 0.5f;
        } else {
            q = 0.f;
        }
        D.geo[2 * dst] = make_float4(a, a, b, b);
        D.geo[2 * dst + 1] = make_float4(c, c, d, d);
        D.qq[dst] = make_float2(q, q);
    };
    if (j < nsrc && !D.culled) {  // records past the live chunks are never read
        float q = 0.f;
        int s = -1;
        if (j < pe) { if (j < ne) { s = D.e_site[j]; q = -1.f; } }
        else if (j < pe + ph) { const int k = j - pe; if (k < nh) { s = D.h_site[k]; q = 1.f; } }
        else if (j < nsrc) { const int k = j - pe - ph; if (k < nd) { s = D.defects[k]; q = (float)D.dq; } }
        record(j, s, q);
    } else if (j < nsrc) {
        // Sorted sources: slot j of the scatter by (class, cell) takes its
        // place at the bin's start plus its rank inside the bin by site (sites
        // are distinct inside a class), shifted to the class's padded start.
        const bool pad = (j >= ne && j < pe) || (j >= pe + nh && j < pe + ph) || j >= pe + ph + nd;
        if (pad) record(j, -1, 0.f);
        if (j < ne + nh + nd) {
            const int i = D.stmp[j];
            const int key = D.skey[i];
            const int lo = key > 0 ? D.sbins[key - 1] : 0, hi = D.sbins[key];
            const int si = src_site(D, i);
            int rank = 0;
            for (int k = lo; k < hi; ++k) rank += src_site(D, D.stmp[k]) < si;
            const int cls = key / (D.ncells + 1);
            const int from = cls == 0 ? 0 : (cls == 1 ? ne : ne + nh);
            const int to = cls == 0 ? 0 : (cls == 1 ? pe : pe + ph);
            record(lo + rank - from + to, si, cls == 0 ? -1.f : (cls == 1 ? 1.f : (float)D.dq));
        }
    }
    if (j < tpad) {
        int s = -1;
        const int g = (D.sorted && j < t) ? D.tperm[j] : j;  // the target in slot j
        if (g < ne) s = D.e_site[g];
        else if (g < ne + nh) s = D.h_site[g - ne];
        else if (g < 2 * ne + nh) s = D.e_f[g - ne - nh];
        else if (g < t) s = D.h_f[g - 2 * ne - nh];
        int x = 0, y = 0, z = 0;
        if (s >= 0) xyz(D, s, x, y, z);  // drain ids decode beyond the lattice: unused
        int slot = 0;
        for (int term = 0; term < 3; ++term) {
            if (!(D.terms & (1u << term))) continue;
            const int xp = term == 0 ? x : (term == 1 ? -1 - x : 2 * D.X - 1 - x);
            // padding slots carry w = -1: left out of the cull's boxes, never read
            D.tgt[(size_t)slot * tpad + j] = make_float4(
                (float)xp, (float)y, (float)z, j < t ? (float)(xp * xp + y * y + z * z) : -1.f);
            ++slot;
        }
    }
}

__device__ __forceinline__ void finalize_body(const Dev& D, const int g) {
    const int t = 2 * (D.cnt[I_NE] + D.cnt[I_NH]);
    const int tpad = D.cnt[I_TPAD], tphys = D.cnt[I_TPHYS];
    if (g >= t) return;
    double v = 0.0, n = 0.0;
    if (D.culled) {
        // the partials of the tile's work items, in item (= chunk) order; the
        // terms' streams read side by side, four items at a time
        const double* qp[3];
        const float* qn[3];
        int ni[3], nmax = 0;
#pragma unroll
        for (int slot = 0; slot < 3; ++slot) {
            ni[slot] = 0;
            qp[slot] = D.part;
            qn[slot] = D.part_norm;
            if (slot < D.nterms) {
                const int p = slot * tpad + g;
                const int tile = p / kCTile, loc = p - tile * kCTile;
                ni[slot] = D.tile_items[tile];
                const size_t f = (size_t)D.tile_first[tile] * kCTile + loc;
                qp[slot] = D.part + f;
                qn[slot] = D.part_norm + f;
                nmax = max(nmax, ni[slot]);
            }
        }
        double s[3] = {0.0, 0.0, 0.0}, m[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < nmax; i += 4) {
            double pv[3][4];
            float nv[3][4];
#pragma unroll
            for (int slot = 0; slot < 3; ++slot)
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const bool on = i + u < ni[slot];
                    pv[slot][u] = on ? qp[slot][(size_t)(i + u) * kCTile] : 0.0;
                    nv[slot][u] = on ? qn[slot][(size_t)(i + u) * kCTile] : 0.f;
                }
#pragma unroll
            for (int slot = 0; slot < 3; ++slot)
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (i + u < ni[slot]) {
                        s[slot] += pv[slot][u];
                        m[slot] += (double)nv[slot][u];
                    }
        }
        v = s[0] - s[1] - s[2];
        n = m[0] + m[1] + m[2];
        const int target = D.tperm[g];
        D.Vt[target] = D.prefactor * v;
        D.Nt[target] = D.prefactor * n;
        return;
    }
    for (int slot = 0; slot < D.nterms; ++slot) {
        double s = 0.0, m = 0.0;
        // four splits' loads in flight, then the adds in split order (same bits)
        int sp = 0;
        for (; sp + 4 <= D.splits; sp += 4) {
            double pv[4];
            float nv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const size_t o = (size_t)(sp + u) * tphys + (size_t)slot * tpad + g;
                pv[u] = D.part[o];
                nv[u] = D.part_norm[o];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                s += pv[u];
                m += (double)nv[u];
            }
        }
        for (; sp < D.splits; ++sp) {
            const size_t o = (size_t)sp * tphys + (size_t)slot * tpad + g;
            s += D.part[o];
            m += (double)D.part_norm[o];
        }
        v = slot == 0 ? s : v - s;
        n += m;
    }
    const int target = D.sorted ? D.tperm[g] : g;  // g is a physical slot
    D.Vt[target] = D.prefactor * v;
    D.Nt[target] = D.prefactor * n;
}

// The counting sort of the step's targets (current sites of electrons and
// holes, then their proposed sites, as pack_body lists them) by the Morton
// rank of their lattice cell; proposed drains go to the last bin.
// Culled replicas sort their sources the same way, keyed by (charge class,
// cell): key = class * (ncells + 1) + cell rank.
__device__ __forceinline__ void tbins_zero_body(const Dev& D, const int i) {
    if (i <= D.ncells) D.bins[i] = 0;
    if (D.culled && i < 3 * (D.ncells + 1)) D.sbins[i] = 0;
}
__device__ __forceinline__ int site_bin(const Dev& D, const int s) {
    if (s < 0 || s >= D.V) return D.ncells;
    int x, y, z;
    xyz(D, s, x, y, z);
    const int sh = D.cell_shift;
    return D.cell_rank[(x >> sh) + D.cells_x * ((y >> sh) + D.cells_y * (z >> sh))];
}
__device__ __forceinline__ void tbins_body(const Dev& D, const int g) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    if (g < 2 * (ne + nh)) {
        int s;
        if (g < ne) s = D.e_site[g];
        else if (g < ne + nh) s = D.h_site[g - ne];
        else if (g < 2 * ne + nh) s = D.e_f[g - ne - nh];
        else s = D.h_f[g - 2 * ne - nh];
        const int b = site_bin(D, s);
        D.tkey[g] = b;
        atomicAdd(&D.bins[b], 1);
    }
    if (D.culled && g < ne + nh + (D.dq != 0 ? D.nd : 0)) {
        const int cls = g < ne ? 0 : (g < ne + nh ? 1 : 2);
        const int key = cls * (D.ncells + 1) + site_bin(D, src_site(D, g));
        D.skey[g] = key;
        atomicAdd(&D.sbins[key], 1);
    }
}
__device__ __forceinline__ void tscatter_body(const Dev& D, const int g) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    if (g < 2 * (ne + nh)) (D.culled ? D.ttmp : D.tperm)[atomicAdd(&D.bins[D.tkey[g]], 1)] = g;
    if (D.culled && g < ne + nh + (D.dq != 0 ? D.nd : 0))
        D.stmp[atomicAdd(&D.sbins[D.skey[g]], 1)] = g;
}
// Culled replicas: the target scattered to slot j goes to its bin's start
// plus its rank inside the bin by index.  A target's sum is split into the
// work items of its tile, so its tile -- and the rounding of the item
// partials' sum -- must not depend on the scatter's order.  D.bins holds the
// bin ends after the scatter.
__device__ __forceinline__ void trank_body(const Dev& D, const int j) {
    if (!D.culled || j >= 2 * (D.cnt[I_NE] + D.cnt[I_NH])) return;
    const int i = D.ttmp[j];
    const int b = D.tkey[i];
    const int lo = b > 0 ? D.bins[b - 1] : 0, hi = D.bins[b];
    int rank = 0;
    for (int k = lo; k < hi; ++k) rank += D.ttmp[k] < i;
    D.tperm[lo + rank] = i;
}

// ChargeAgent::bindingPotential (chargeagent.cpp:463-481)
__device__ __forceinline__ double binding(const Dev& D, bool e, int site) {
    if (e) return D.ht[site] == T_HOLE ? D.sI100 + D.exciton_binding : 0.0;
    return D.et[site] == T_ELECTRON ? D.sI100 - D.exciton_binding : 0.0;
}

__device__ __forceinline__ double coupling_of(const Dev& D, int s, int f) {
    int x0, y0, z0, x1, y1, z1;
    xyz(D, s, x0, y0, z0);
    xyz(D, f, x1, y1, z1);
    const int dx = abs(x0 - x1), dy = abs(y0 - y1), dz = abs(z0 - z1);
    const int h = D.hr + 1;
    return D.coupling[(dx * h + dy) * h + dz];
}

// Random::metropolisWithCoupling (rand.cpp:91-106) on an FP64 energy.
__device__ __forceinline__ bool metropolis(double pd, double beta, double c, double u) {
    if (pd > 0.0) return c * exp(-pd * beta) > u;
    return c > u;
}

__device__ __forceinline__ void decide_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    const uint32_t step = (uint32_t)D.cnt[I_STEP];
    if (i >= ne + nh) return;
    const bool e = i < ne;
    const int k = e ? i : i - ne;
    const int site = e ? D.e_site[k] : D.h_site[k];
    int f = e ? D.e_f[k] : D.h_f[k];
    uint8_t type = (e ? D.et : D.ht)[f];
    // extension: a carrier may not enter the other phase (treated as occupied)
    if (D.confine && f < D.V && type == T_EMPTY && D.phase[f] != (e ? 1 : 0)) type = T_DEFECT;
    const double q = e ? -1.0 : 1.0;
    int32_t out = O_OCCUPIED;
    uint8_t acc = 0;
    double de = 0.0;
    if (type == T_EMPTY) {
        const double c = coupling_of(D, site, f);
        const Philox4 r = draw(D, step, (uint32_t)k, e ? RNG_DECIDE_E : RNG_DECIDE_H);
        const double u = unit_double(r.w[0], r.w[1]);
        double pd = (D.pot[f] - D.pot[site]) * q;
        bool flag = false;
        if (D.coulomb) {
            const int t = ne + nh;
            const double p1 = D.Vt[i] + binding(D, e, site);
            const double p2 = D.Vt[t + i] - D.sI100 * q + binding(D, e, f);
            de = q * (p2 - p1);
            pd += de;
            if (u < c) {
                const double tau = log(c / u) / D.beta;
                const double g = D.guard * (D.Nt[i] + D.Nt[t + i]) + 1e-12 * (1.0 + fabs(pd));
                if (fabs(pd - tau) <= g) flag = true;
                else acc = pd < tau;
            }
        } else {
            acc = metropolis(pd, D.beta, c, u);
        }
        if (flag) {
            const int slot = atomicAdd(&D.cnt[I_NFLAG], 1);
            D.flagged[slot] = i;
            out = -1;  // pending
        } else {
            out = acc ? O_MET_ACCEPT : O_MET_REJECT;
        }
    } else if (type == T_DRAIN) {
        const int which = f - D.V;
        const int agent = e ? (which == E_DRAIN_L ? 0 : 1) : (which == H_DRAIN_L ? 2 : 3);
        atomicAdd(&D.ctr[2 * (4 + agent)], 1ull);
        const Philox4 r = draw(D, step, (uint32_t)k, e ? RNG_DECIDE_E : RNG_DECIDE_H);
        const double u = unit_double(r.w[0], r.w[1]);
        if (D.rate_drain[agent] > u) {  // chooseYes (fluxagent.cpp:125-130)
            atomicAdd(&D.ctr[2 * (4 + agent) + 1], 1ull);
            acc = 1;
            out = O_DRAIN_ACCEPT;
        } else {
            out = O_DRAIN_REJECT;
        }
    }
    D.outcome[i] = out;
    D.de[i] = de;
    D.accept[i] = acc;
}

// FP64 re-evaluation of queued decisions: the potentials at the current and
// future site summed in double over all charges (and their images), then the
// reference's test on the FP64 energy.  One block per queued decision,
// grid-stride over the queue.
// One decision's FP64 sums spread over 32 warps: 1024-thread blocks measured
// faster than 256 for a single replica (256x256x16, 20,922 carriers: step
// 0.646 -> 0.620 ms) and for a batch of 512 uneven replicas (2.27 -> 2.20 ms).
constexpr int kGuardThreads = 1024;
// Each queued decision's source range is cut into this many splits, one
// block each; the block that completes a decision last adds the splits'
// partials in split order (a fixed order) and decides.
constexpr int kGuardSplits = 16;
// Blocks per replica of the batched guard: flagged decisions of one replica
// are spread over them (a replica with M charges flags ~1e-3 M per step).
constexpr int kGuardBlocksPerReplica = 48;
// The batch's guard blocks: most replicas flag no decision in a step, and a
// block with nothing to do costs its launch and retirement, so they are
// small; a replica gets one block per 512 charges of capacity.
constexpr int kGuardThreadsBatch = 256;
// Indices per thread of the batched element-wise kernels (see LGM_BATCH_LOOP).
constexpr int kItemsPerThread = 4;

// FP64 potentials at two sites in one pass over the sources (the guard's
// re-evaluation): the same cutoff and image rules as the pair kernel, terms
// w(r^2) from the FP64 table (1/sqrt(k) or erf(f sqrt(k))/sqrt(k), computed on
// the host in IEEE double), summed per thread and then across the block.
__device__ double2 fp64_potential2(const Dev& D, int ne, int nh, int site_a, int site_b, int j0,
                                   int j1, double2* red) {
    int xa, ya, za, xb, yb, zb;
    xyz(D, site_a, xa, ya, za);
    xyz(D, site_b, xb, yb, zb);
    double acc_a = 0.0, acc_b = 0.0;
    for (int j = j0 + (int)threadIdx.x; j < j1; j += blockDim.x) {
        int s;
        double q;
        if (j < ne) { s = D.e_site[j]; q = -1.0; }
        else if (j < ne + nh) { s = D.h_site[j - ne]; q = 1.0; }
        else { s = D.defects[j - ne - nh]; q = (double)D.dq; }
        int xj, yj, zj;
        xyz(D, s, xj, yj, zj);
        const int dya = ya - yj, dza = za - zj, dyb = yb - yj, dzb = zb - zj;
        const int ra = dya * dya + dza * dza, rb = dyb * dyb + dzb * dzb;
        for (int term = 0; term < 3; ++term) {
            if (!(D.terms & (1u << term))) continue;
            const int dxa = term == 0 ? xa - xj : (term == 1 ? xa + xj + 1 : 2 * D.X - 1 - xa - xj);
            const int dxb = term == 0 ? xb - xj : (term == 1 ? xb + xj + 1 : 2 * D.X - 1 - xb - xj);
            const int r2a = dxa * dxa + ra, r2b = dxb * dxb + rb;
            const double qs = term == 0 ? q : -q;
            if (r2a > 0 && r2a < D.cutoff2) acc_a += qs * D.w64[r2a];
            if (r2b > 0 && r2b < D.cutoff2) acc_b += qs * D.w64[r2b];
        }
    }
    // Warp sums by shuffles, then the warp sums by warp 0 (a fixed order;
    // blockDim a multiple of 32, red holds at least 32 entries).
    for (int o = 16; o > 0; o >>= 1) {
        acc_a += __shfl_down_sync(0xffffffffu, acc_a, o);
        acc_b += __shfl_down_sync(0xffffffffu, acc_b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) red[warp] = make_double2(acc_a, acc_b);
    __syncthreads();
    if (warp == 0) {
        double2 t = lane < nw ? red[lane] : make_double2(0.0, 0.0);
        for (int o = 16; o > 0; o >>= 1) {
            t.x += __shfl_down_sync(0xffffffffu, t.x, o);
            t.y += __shfl_down_sync(0xffffffffu, t.y, o);
        }
        __syncwarp();
        if (lane == 0) red[0] = t;
    }
    __syncthreads();
    const double2 v = red[0];
    __syncthreads();
    return v;
}

__device__ __forceinline__ void guard_body(const Dev& D, const int block, const int nblocks,
                                           double2* red) {
    __shared__ int s_last;
    const int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    const int nflag = D.cnt[I_NFLAG];
    const uint32_t step = (uint32_t)D.cnt[I_STEP];
    const int n = ne + nh + (D.dq != 0 ? D.nd : 0);
    for (int w = block; w < nflag * kGuardSplits; w += nblocks) {
        const int q_i = w / kGuardSplits, sp = w - q_i * kGuardSplits;
        const int i = D.flagged[q_i];
        const bool e = i < ne;
        const int k = e ? i : i - ne;
        const int site = e ? D.e_site[k] : D.h_site[k];
        const int f = e ? D.e_f[k] : D.h_f[k];
        const double q = e ? -1.0 : 1.0;
        const int j0 = (int)((long long)sp * n / kGuardSplits);
        const int j1 = (int)((long long)(sp + 1) * n / kGuardSplits);
        const double2 part = fp64_potential2(D, ne, nh, site, f, j0, j1, red);
        if (threadIdx.x == 0) {
            D.gpart[(size_t)q_i * kGuardSplits + sp] = part;
            __threadfence();
            s_last = atomicAdd(&D.gdone[q_i], 1) == kGuardSplits - 1;
        }
        __syncthreads();
        if (s_last && threadIdx.x == 0) {
            __threadfence();
            double2 t = make_double2(0.0, 0.0);
            for (int u = 0; u < kGuardSplits; ++u) {  // split order
                const double2 p = __ldcg(&D.gpart[(size_t)q_i * kGuardSplits + u]);
                t.x += p.x;
                t.y += p.y;
            }
            D.gdone[q_i] = 0;
            const double v1 = D.prefactor * t.x, v2 = D.prefactor * t.y;
            const double p1 = v1 + binding(D, e, site);
            const double p2 = v2 - D.sI100 * q + binding(D, e, f);
            const double de = q * (p2 - p1);
            double pd = (D.pot[f] - D.pot[site]) * q;
            pd += de;
            const Philox4 r = draw(D, step, (uint32_t)k, e ? RNG_DECIDE_E : RNG_DECIDE_H);
            const double u = unit_double(r.w[0], r.w[1]);
            const bool acc = metropolis(pd, D.beta, coupling_of(D, site, f), u);
            D.outcome[i] = acc ? O_MET_ACCEPT : O_MET_REJECT;
            D.accept[i] = acc;
            D.de[i] = de;
            atomicAdd(&D.ctr[C_GUARD], 1ull);
        }
        __syncthreads();  // s_last is read before the next decision writes it
    }
}

// completeTick, part 1: contested empty sites go to the lowest list index.
__device__ __forceinline__ void claim_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    if (i >= ne + nh || !D.accept[i]) return;
    const bool e = i < ne;
    const int k = e ? i : i - ne;
    if ((e ? D.e_rm : D.h_rm)[k]) return;  // recombined: completeTick only unregisters
    const int f = e ? D.e_f[k] : D.h_f[k];
    if (f < D.V) atomicMin(&(e ? D.claim_e : D.claim_h)[f], k);
}

// completeTick, part 2: winners move, drains remove (site marked -1).
__device__ __forceinline__ void move_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    unsigned long long moved = 0, props = 0;
    if (i < ne + nh) {
        props = 1;
        const bool e0 = i < ne;
        const int k0 = e0 ? i : i - ne;
        if ((e0 ? D.e_rm : D.h_rm)[k0]) {
            // recombined: leave the lattice (chargeagent.cpp:166-170)
            int32_t* sites = e0 ? D.e_site : D.h_site;
            (e0 ? D.et : D.ht)[sites[k0]] = T_EMPTY;
            sites[k0] = -1;
            D.cnt[I_REMOVED] = 1;
            atomicMin(&D.cnt[e0 ? I_FIRST_E : I_FIRST_H], k0);
        } else if (D.accept[i]) {
            const bool e = i < ne;
            const int k = e ? i : i - ne;
            int32_t* sites = e ? D.e_site : D.h_site;
            uint8_t* own = e ? D.et : D.ht;
            const int s = sites[k];
            const int f = (e ? D.e_f : D.h_f)[k];
            if (f >= D.V) {
                own[s] = T_EMPTY;
                sites[k] = -1;
                D.cnt[I_REMOVED] = 1;
                atomicMin(&D.cnt[e ? I_FIRST_E : I_FIRST_H], k);
                moved = 1;
            } else if ((e ? D.claim_e : D.claim_h)[f] == k) {
                own[s] = T_EMPTY;
                own[f] = e ? T_ELECTRON : T_HOLE;
                sites[k] = f;
                moved = 1;
            }
        }
    }
    // warp-aggregated counters
    for (int o = 16; o > 0; o >>= 1) {
        moved += __shfl_down_sync(0xffffffffu, moved, o);
        props += __shfl_down_sync(0xffffffffu, props, o);
    }
    if ((threadIdx.x & 31) == 0 && props) {
        atomicAdd(&D.ctr[C_PROPOSALS], props);
        if (moved) atomicAdd(&D.ctr[C_ACCEPTED], moved);
    }
}

__device__ __forceinline__ void unclaim_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    if (i >= ne + nh || !D.accept[i]) return;
    const bool e = i < ne;
    const int k = e ? i : i - ne;
    if ((e ? D.e_rm : D.h_rm)[k]) return;
    const int f = e ? D.e_f[k] : D.h_f[k];
    if (f < D.V) (e ? D.claim_e : D.claim_h)[f] = INT_MAX;
}

// RecombinationAgent::tryToAccept for every electron (drainagent.cpp:113-214).
// The reference walks the electrons in list order and skips a hole already
// removed by an earlier electron; here every electron draws its candidate and
// its acceptance from its own counter, and the lowest-index successful electron
// of each hole is the one that removes it -- the same outcome.
__device__ __forceinline__ void hmap_body(const Dev& D, const int k, const bool set) {
    if (k < D.cnt[I_NH0]) D.h_at[D.h_site[k]] = set ? k : -1;
}

__device__ __forceinline__ void recomb_propose_body(const Dev& D, const int i) {
    const int ne = D.cnt[I_NE0];
    if (i >= ne) return;
    D.e_rch[i] = -1;
    const int site = D.e_site[i];
    int cand[48];
    int n = 0;
    if (D.ht[site] == T_HOLE) cand[n++] = site;
    if (D.rec_range > 0) {
        int nb[40];
        const int m = neighbors(D, site, true, nb, D.rec_range);
        for (int j = 0; j < m; ++j)
            if (D.ht[nb[j]] == T_HOLE) cand[n++] = nb[j];
    }
    if (n == 0) return;
    const Philox4 r = draw(D, (uint32_t)D.cnt[I_STEP], (uint32_t)i, RNG_RECOMB);
    const int hk = D.h_at[cand[uint_below(r.w[0], (uint32_t)n)]];
    D.e_rch[i] = hk;
    if (D.rec_rate > unit_double(r.w[1], r.w[2])) atomicMin(&D.rclaim[hk], i);
}

__device__ __forceinline__ void recomb_resolve_body(const Dev& D, const int i) {
    if (i >= D.cnt[I_NE0]) return;
    const int hk = D.e_rch[i];
    if (hk < 0) return;
    const int w = D.rclaim[hk];
    if (w == INT_MAX || i <= w) atomicAdd(&D.ctr[C_RECOMB], 1ull);  // hole still there
    if (i == w) {
        atomicAdd(&D.ctr[C_RECOMB + 1], 1ull);
        D.e_rm[i] = 1;
        D.h_rm[hk] = 1;
    }
}

__device__ __forceinline__ void recomb_reset_body(const Dev& D, const int i) {
    if (i < D.cnt[I_NE0] && D.e_rch[i] >= 0) D.rclaim[D.e_rch[i]] = INT_MAX;
    hmap_body(D, i, false);
}

// Stable removal of drained carriers (Simulation::nextTick removeAt), then the
// electrode sources (simulation.cpp:246-249) and currentStep += 1.  One block.
constexpr int kCompactThreads = 1024;

// Entries before `start` are all kept (no removal below it) and stay put.
constexpr int kCompactPer = 8;  // consecutive list entries per thread and round
__device__ int compact(int32_t* a, int n, int* warp_sums, int start) {
    start = min(max(start, 0), n);
    int base = start;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    const int span = (int)blockDim.x * kCompactPer;
    for (int t0 = start; t0 < n; t0 += span) {
        // Every read of the round precedes every write (two barriers apart),
        // and an entry only moves to a lower index inside the rounds read so
        // far, so the compaction runs in place.
        const int i0 = t0 + (int)threadIdx.x * kCompactPer;
        int v[kCompactPer];
        int cnt = 0;
#pragma unroll
        for (int u = 0; u < kCompactPer; ++u) {
            v[u] = i0 + u < n ? a[i0 + u] : -1;
            cnt += v[u] >= 0;
        }
        int inc = cnt;  // inclusive scan over the warp, then over the warps
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) warp_sums[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            int w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < nw) warp_sums[lane] = w;
        }
        __syncthreads();
        int pos = base + (warp > 0 ? warp_sums[warp - 1] : 0) + inc - cnt;
        const int total = warp_sums[nw - 1];
#pragma unroll
        for (int u = 0; u < kCompactPer; ++u)
            if (v[u] >= 0) a[pos++] = v[u];
        base += total;
        __syncthreads();  // warp_sums is read before the next round writes it
    }
    return base;
}

// Potential::coulombE/H/D or coulombImageE/H/D (potential.cpp:351-415,
// 483-547, 615-683) at one site: point charges q at `sites`, direct or the
// image in the left electrode (x distance x_i + x_j + 1), 1/r in FP64 as the
// reference's iR table holds it (1.0 / sqrt(r^2)), times the prefactor.  The
// whole block takes part; the partial sums are added in a fixed order.
__device__ double block_species_potential(const Dev& D, int site, const int32_t* sites, int n,
                                          double q, bool image, double* red) {
    int xi, yi, zi;
    xyz(D, site, xi, yi, zi);
    double acc = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        int xj, yj, zj;
        xyz(D, sites[j], xj, yj, zj);
        const int dx = image ? xi + xj + 1 : xi - xj, dy = yi - yj, dz = zi - zj;
        const int r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0 && r2 < D.cutoff2) {
            const double w = 1.0 / sqrt((double)r2);
            acc = image ? acc - w * q : acc + w * q;
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    double total = 0.0;
    for (int w = 0; w < nw; ++w) total += red[w];
    __syncthreads();
    return total * D.prefactor;
}

// Block-shared state of the injection phase.
struct InjectState {
    int ne, nh, site, valid;
    double u;
};

// SourceAgent::tryToInject (sourceagent.cpp:92-103) for electrode source s
// (0 eL, 1 eR, 2 hL, 3 hR) on the draw at {step, index, purpose}: the site
// from the face, validToInject (sourceagent.cpp:192-232), then shouldTransport
// (sourceagent.cpp:168-181): chooseYes on the rate, or with source.metropolis
// metropolisWithCoupling on energyChange (sourceagent.cpp:125-161), which with
// source.coulomb adds the Coulomb and left-image sums at the site (the
// source's own potential is 0).  Every thread of the block calls it.
__device__ void block_try_inject(const Dev& D, InjectState& S, int s, uint32_t step,
                                 uint32_t index, uint32_t purpose, double* red) {
    const bool e = s < 2, left = (s % 2) == 0;
    if (threadIdx.x == 0) {
        D.ctr[2 * s] += 1;  // attempts (sourceagent.cpp:94)
        const Philox4 r = draw(D, step, index, purpose);
        const int idx = (int)uint_below(r.w[0], (uint32_t)(D.Y * D.Z));
        const int site = D.X * idx + (left ? 0 : D.X - 1);
        const uint8_t* own = e ? D.et : D.ht;
        const int count = e ? S.ne : S.nh;
        const int cap = e ? D.cap_e : D.cap_h;
        S.site = site;
        S.valid = count < cap && D.rate_src[s] > 0 && own[site] == T_EMPTY;
        S.u = unit_double(r.w[1], r.w[2]);
    }
    __syncthreads();
    if (!S.valid) return;
    const int site = S.site;
    double de = 0.0;
    if (D.src_metro) {
        double p2 = D.pot[site];
        if (D.src_coulomb) {
            // p2 += coulombH + coulombImageH + coulombE + coulombImageE (+ D)
            p2 += block_species_potential(D, site, D.h_site, S.nh, 1.0, false, red);
            p2 += block_species_potential(D, site, D.h_site, S.nh, 1.0, true, red);
            p2 += block_species_potential(D, site, D.e_site, S.ne, -1.0, false, red);
            p2 += block_species_potential(D, site, D.e_site, S.ne, -1.0, true, red);
            if (D.dq != 0) {
                p2 += block_species_potential(D, site, D.defects, D.nd, (double)D.dq, false, red);
                p2 += block_species_potential(D, site, D.defects, D.nd, (double)D.dq, true, red);
            }
        }
        de = e ? 0.0 - p2 : p2 - 0.0;
    }
    if (threadIdx.x == 0) {
        const double rate = D.rate_src[s];
        const bool accept = D.src_metro ? metropolis(de, D.beta, rate, S.u) : rate > S.u;
        if (accept) {
            D.ctr[2 * s + 1] += 1;
            (e ? D.et : D.ht)[site] = e ? T_ELECTRON : T_HOLE;
            if (e) D.e_site[S.ne++] = site;
            else D.h_site[S.nh++] = site;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void compact_inject_body(const Dev& D, int* warp_sums, double* red) {
    __shared__ InjectState S;
    int ne = D.cnt[I_NE0], nh = D.cnt[I_NH0];
    if (D.cnt[I_REMOVED]) {
        ne = compact(D.e_site, ne, warp_sums, D.cnt[I_FIRST_E]);
        nh = compact(D.h_site, nh, warp_sums, D.cnt[I_FIRST_H]);
    }
    const uint32_t step = (uint32_t)D.cnt[I_STEP];
    if (threadIdx.x == 0) {
        S.ne = ne;
        S.nh = nh;
    }
    __syncthreads();
    if (D.solar) {
        if (threadIdx.x == 0) {
            // ExcitonSourceAgent::tryToInject (sourceagent.cpp:92-103, 120-123, 234-250)
            D.ctr[C_XSRC] += 1;
            const Philox4 r = draw(D, step, 0u, RNG_EXCITON);
            const int nb = D.cnt[I_NBONDS];
            int es, hs;
            if (D.gen_iface && nb > 0) {
                const uint32_t b = uint_below(r.w[0], (uint32_t)nb);
                hs = D.bonds[2 * b];
                es = D.bonds[2 * b + 1];
            } else {
                es = hs = (int)uint_below(r.w[0], (uint32_t)D.V);
            }
            const bool valid = S.ne < D.cap_e && S.nh < D.cap_h && D.gen_rate > 0 &&
                               D.et[es] == T_EMPTY && D.ht[hs] == T_EMPTY;
            if (valid && D.gen_rate > unit_double(r.w[1], r.w[2])) {
                D.ctr[C_XSRC + 1] += 1;
                D.et[es] = T_ELECTRON;
                D.ht[hs] = T_HOLE;
                D.e_site[S.ne++] = es;
                D.h_site[S.nh++] = hs;
            }
        }
        __syncthreads();
        if (D.balance) {
            // Simulation::balanceCharges (simulation.cpp:253-353): electrons
            // from the electrode on the low-potential side until they are no
            // fewer than the holes, then holes alike; a uniform draw picks
            // the side when the voltages are equal
            for (int species = 0; species < 2; ++species) {
                const bool e = species == 0;
                const uint32_t purpose = e ? RNG_BALANCE_E : RNG_BALANCE_H;
                for (int t = 0;; ++t) {
                    const int more = e ? S.nh - S.ne : S.ne - S.nh;
                    const bool at_max = e ? S.ne >= D.cap_e : S.nh >= D.cap_h;
                    if (more <= 0 || at_max) break;
                    if (t >= kBalanceTries) {  // the reference stops with a fatal error
                        if (threadIdx.x == 0) atomicOr(D.err, DEVERR_STATE);
                        break;
                    }
                    bool left;
                    if (D.volt_r > D.volt_l) left = e;
                    else if (D.volt_l > D.volt_r) left = !e;
                    else {
                        const Philox4 r = draw(D, step, (uint32_t)t, purpose + 1);
                        const bool above = unit_double(r.w[0], r.w[1]) > 0.5;
                        left = e ? above : !above;
                    }
                    block_try_inject(D, S, (e ? 0 : 2) + (left ? 0 : 1), step, (uint32_t)t,
                                     purpose, red);
                }
            }
        }
    } else {
        // the electrode sources in the reference's order (simulation.cpp:246-249)
        for (int s = 0; s < 4; ++s) block_try_inject(D, S, s, step, 0u, RNG_SOURCE + (uint32_t)s, red);
    }
    if (threadIdx.x == 0) {
        D.cnt[I_NE] = S.ne;
        D.cnt[I_NH] = S.nh;
        D.cnt[I_STEP] = (int32_t)(step + 1);
    }
}

// Single-replica kernels: the Dev travels by value.
#define LGM_THREAD_INDEX (int)(blockIdx.x * blockDim.x + threadIdx.x)
__global__ void k_choose(Dev D) {
    pdl_wait();
    pdl_trigger(); choose_body(D, LGM_THREAD_INDEX); }
__global__ void k_pack(Dev D) {
    pdl_wait();
    pdl_trigger(); pack_body(D, LGM_THREAD_INDEX); }
__global__ void k_finalize(Dev D) {
    pdl_wait();
    pdl_trigger(); finalize_body(D, LGM_THREAD_INDEX); }
// finalize_body's culled branch with a block of 32 x 3 threads per 32
// targets: warp y sums term slot y's item partials (and norms) in item order,
// eight items in flight, and warp 0 combines the slots -- the same sums in
// the same order, three times the threads.
__global__ void __launch_bounds__(96) k_finalize_culled(Dev D) {
    pdl_wait();
    pdl_trigger();
    constexpr int kRows = 8;
    __shared__ double s_v[3][32], s_n[3][32];
    const int t = 2 * (D.cnt[I_NE] + D.cnt[I_NH]);
    const int tpad = D.cnt[I_TPAD];
    const int x = (int)threadIdx.x, slot = (int)threadIdx.y;
    const int g = (int)blockIdx.x * 32 + x;
    double sv = 0.0, sn = 0.0;
    if (g < t && slot < D.nterms) {
        const int p = slot * tpad + g;
        const int tile = p / kCTile, loc = p - tile * kCTile;
        const int ni = D.tile_items[tile];
        const size_t f = (size_t)D.tile_first[tile] * kCTile + loc;
        for (int i = 0; i < ni; i += kRows) {
            double pv[kRows];
            float nv[kRows];
#pragma unroll
            for (int u = 0; u < kRows; ++u) {
                const bool on = i + u < ni;
                pv[u] = on ? D.part[f + (size_t)(i + u) * kCTile] : 0.0;
                nv[u] = on ? D.part_norm[f + (size_t)(i + u) * kCTile] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kRows; ++u)
                if (i + u < ni) {
                    sv += pv[u];
                    sn += (double)nv[u];
                }
        }
    }
    s_v[slot][x] = sv;
    s_n[slot][x] = sn;
    __syncthreads();
    if (slot == 0 && g < t) {
        const double v = s_v[0][x] - s_v[1][x] - s_v[2][x];
        const double n = s_n[0][x] + s_n[1][x] + s_n[2][x];
        const int target = D.tperm[g];
        D.Vt[target] = D.prefactor * v;
        D.Nt[target] = D.prefactor * n;
    }
}
__global__ void k_decide(Dev D) {
    pdl_wait();
    pdl_trigger(); decide_body(D, LGM_THREAD_INDEX); }
__global__ void k_tbins_zero(Dev D) {
    pdl_wait();
    pdl_trigger(); tbins_zero_body(D, LGM_THREAD_INDEX); }
__global__ void k_tbins(Dev D) {
    pdl_wait();
    pdl_trigger(); tbins_body(D, LGM_THREAD_INDEX); }
__global__ void __launch_bounds__(1024) k_tbins_scan(Dev D) {
    pdl_wait();
    pdl_trigger();
    if (blockIdx.x == 0) block_exclusive_scan(D.bins, D.ncells + 1);
    else block_exclusive_scan(D.sbins, 3 * (D.ncells + 1));
}
// Source records and work list of the culled pair sum (lgm_cull.cuh).
__host__ __device__ __forceinline__ PairArgs pair_args(const Dev& D) {
    PairArgs A;
    A.geo = D.geo; A.qq = D.qq; A.splits = D.splits; A.tgt = D.tgt; A.part = D.part;
    A.part_norm = D.part_norm;
    A.c2 = (float)D.cutoff2; A.tab = D.gtab; A.tab_k = D.gauss ? D.gtab_k : 0;
    A.err = D.err; A.dyn = D.cnt + I_NCHUNK;  // dyn[0] = n_chunks, dyn[1] = t_phys
    return A;
}
__host__ __device__ __forceinline__ CullArgs cull_args(const Dev& D) {
    CullArgs C;
    C.cbox = D.cbox; C.gbox = D.gbox;
    C.tgt = D.tgt; C.dyn = D.cnt + I_NCHUNK;
    C.c2 = D.cutoff2; C.tile_size = kCTile;
    C.per_item = kCullPerItem; C.max_items = D.max_items;
    C.live = D.live; C.live_stride = D.src_cap / CH;
    C.items = D.items; C.item_count = D.item_count; C.work = D.item_count + 1;
    C.tile_first = D.tile_first; C.tile_items = D.tile_items;
    // costs from the pair kernel's warp segments; a standalone replica orders
    // its own items (a batch orders all its culled replicas' items at once)
    C.warp_targets = 64 * kCRP;
    C.hist = D.chist;
    C.order = D.corder;
    C.done = D.item_count + 2;
    return C;
}
__global__ void __launch_bounds__(CH) k_chunk_boxes(Dev D) {
    pdl_wait();
    pdl_trigger();
    chunk_boxes_body(pair_args(D), cull_args(D), (int)blockIdx.x);
}
__global__ void __launch_bounds__(kCullThreads) k_cull(Dev D) {
    pdl_wait();
    pdl_trigger(); cull_body(cull_args(D), (int)blockIdx.x); }
__global__ void k_tscatter(Dev D) {
    pdl_wait();
    pdl_trigger(); tscatter_body(D, LGM_THREAD_INDEX); }
__global__ void k_trank(Dev D) {
    pdl_wait();
    pdl_trigger(); trank_body(D, LGM_THREAD_INDEX); }
__global__ void __launch_bounds__(kGuardThreads) k_guard(Dev D) {
    pdl_wait();
    pdl_trigger();
    __shared__ double2 red[32];
    guard_body(D, blockIdx.x, gridDim.x, red);
}
__global__ void k_hmap(Dev D) {
    pdl_wait();
    pdl_trigger(); hmap_body(D, LGM_THREAD_INDEX, true); }
__global__ void k_recomb_propose(Dev D) {
    pdl_wait();
    pdl_trigger(); recomb_propose_body(D, LGM_THREAD_INDEX); }
__global__ void k_recomb_resolve(Dev D) {
    pdl_wait();
    pdl_trigger(); recomb_resolve_body(D, LGM_THREAD_INDEX); }
__global__ void k_recomb_reset(Dev D) {
    pdl_wait();
    pdl_trigger(); recomb_reset_body(D, LGM_THREAD_INDEX); }
__global__ void k_claim(Dev D) {
    pdl_wait();
    pdl_trigger(); claim_body(D, LGM_THREAD_INDEX); }
__global__ void k_move(Dev D) {
    pdl_wait();
    pdl_trigger(); move_body(D, LGM_THREAD_INDEX); }
__global__ void k_unclaim(Dev D) {
    pdl_wait();
    pdl_trigger(); unclaim_body(D, LGM_THREAD_INDEX); }
__global__ void __launch_bounds__(kCompactThreads) k_compact_inject(Dev D) {
    pdl_wait();
    pdl_trigger();
    __shared__ int warp_sums[32];
    __shared__ double red[32];
    compact_inject_body(D, warp_sums, red);
}

// Batched kernels: block b works for replica map[b].x as its local block
// map[b].y of map[b].z blocks, over indices [0, map[b].w) of that replica with
// a block-uniform stride (every block lies inside one replica, so warp-level
// sums stay within a replica, and every thread of a block runs the same number
// of iterations).  A replica gets one block per kItemsPerThread * 256 indices
// of its capacity, so small replicas in a big batch cost few idle blocks.
#define LGM_BATCH_LOOP(CALL)                                                          \
    const int4 m = map[blockIdx.x];                                                   \
    const Dev& D = R[m.x];                                                            \
    for (int base = m.y * (int)blockDim.x; base < m.w; base += m.z * (int)blockDim.x) { \
        const int i = base + (int)threadIdx.x;                                        \
        CALL;                                                                         \
    }
__global__ void kb_choose(const Dev* R, const int4* map) { LGM_BATCH_LOOP(choose_body(D, i)) }
__global__ void kb_pack(const Dev* R, const int4* map) { LGM_BATCH_LOOP(pack_body(D, i)) }
__global__ void kb_finalize(const Dev* R, const int4* map) { LGM_BATCH_LOOP(finalize_body(D, i)) }
__global__ void kb_decide(const Dev* R, const int4* map) { LGM_BATCH_LOOP(decide_body(D, i)) }
__global__ void kb_tbins_zero(const Dev* R, const int4* map) { LGM_BATCH_LOOP(tbins_zero_body(D, i)) }
__global__ void kb_tbins(const Dev* R, const int4* map) { LGM_BATCH_LOOP(tbins_body(D, i)) }
__global__ void kb_tscatter(const Dev* R, const int4* map) { LGM_BATCH_LOOP(tscatter_body(D, i)) }
__global__ void kb_trank(const Dev* R, const int4* map) { LGM_BATCH_LOOP(trank_body(D, i)) }
// one block per replica of the list; a second row scans culled replicas' source bins
__global__ void __launch_bounds__(1024) kb_tbins_scan(const Dev* R, const int* list) {
    const Dev& D = R[list[blockIdx.x]];
    if (blockIdx.y == 0) block_exclusive_scan(D.bins, D.ncells + 1);
    else if (D.culled) block_exclusive_scan(D.sbins, 3 * (D.ncells + 1));
}
// The culled replicas' chunk boxes and tile culls: block b works for replica
// map[b].x as its chunk or tile map[b].y.
__global__ void __launch_bounds__(CH) kb_chunk_boxes(const Dev* R, const int2* map) {
    const Dev& D = R[map[blockIdx.x].x];
    chunk_boxes_body(pair_args(D), cull_args(D), map[blockIdx.x].y);
}
__global__ void __launch_bounds__(kCullThreads) kb_cull(const Dev* R, const int2* map) {
    cull_body(cull_args(R[map[blockIdx.x].x]), map[blockIdx.x].y);
}
// Pairs the work-item kernel tests for the per-phase replicas that do not
// cull: every physical target against every packed source (one block).
__global__ void kb_tested_pairs(const Dev* R, const int* list, int n, unsigned long long* out) {
    for (int i = (int)threadIdx.x; i < n; i += (int)blockDim.x) {
        const Dev& D = R[list[i]];
        if (D.culled) continue;
        const int32_t* dyn = D.cnt + I_NCHUNK;
        atomicAdd(out, (unsigned long long)dyn[0] * CH * (unsigned long long)dyn[1]);
    }
}
// One block, after the culls: offs[i] = work items of culled replicas
// list[0 .. i-1] (i <= n) and offs[n + 1] = 0, the next item to take
// (ProblemList::work); then order[] = all those items, numbered as
// ProblemList numbers them, by decreasing cost (the batch's histogram).
__global__ void __launch_bounds__(1024) kb_item_order(ProblemList L, const Dev* R,
                                                      const int32_t* hist, int32_t* offs,
                                                      int32_t* order) {
    __shared__ int s_off[kCostBuckets];
    const int n = L.n;
    for (int i = (int)threadIdx.x; i <= n; i += (int)blockDim.x)
        offs[i] = i < n ? *R[L.list[i]].item_count : 0;
    for (int b = (int)threadIdx.x; b < kCostBuckets; b += (int)blockDim.x) s_off[b] = hist[b];
    __syncthreads();
    block_exclusive_scan(offs, n + 1);
    if (threadIdx.x == 0) offs[n + 1] = 0;
    // the offsets in shared memory for the items' replica searches (up to
    // kOffsInShared replicas; more search global memory)
    constexpr int kOffsInShared = 2048;
    __shared__ int s_offs[kOffsInShared];
    const bool in_smem = n + 1 <= kOffsInShared;
    if (in_smem)
        for (int i = (int)threadIdx.x; i <= n; i += (int)blockDim.x) s_offs[i] = offs[i];
    cost_offsets(s_off);  // (its barriers also publish s_offs)
    const int* so = in_smem ? s_offs : offs;
    const int total = so[n];
    for (int g = (int)threadIdx.x; g < total; g += (int)blockDim.x) {
        int lo = 0, hi = n;  // the last replica whose first item is at or before g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (so[mid] <= g) lo = mid;
            else hi = mid;
        }
        const int c = min(L.C(L.list[lo]).items[g - so[lo]].w, kCostBuckets - 1);
        order[atomicAdd(&s_off[c], 1)] = g;
    }
}
__global__ void __launch_bounds__(kGuardThreadsBatch) kb_guard(const Dev* R, const int4* map) {
    __shared__ double2 red[32];
    const int4 m = map[blockIdx.x];
    guard_body(R[m.x], m.y, m.z, red);
}
__global__ void kb_hmap(const Dev* R, const int4* map) { LGM_BATCH_LOOP(hmap_body(D, i, true)) }
__global__ void kb_recomb_propose(const Dev* R, const int4* map) {
    LGM_BATCH_LOOP(recomb_propose_body(D, i))
}
__global__ void kb_recomb_resolve(const Dev* R, const int4* map) {
    LGM_BATCH_LOOP(recomb_resolve_body(D, i))
}
__global__ void kb_recomb_reset(const Dev* R, const int4* map) {
    LGM_BATCH_LOOP(recomb_reset_body(D, i))
}
__global__ void kb_claim(const Dev* R, const int4* map) { LGM_BATCH_LOOP(claim_body(D, i)) }
__global__ void kb_move(const Dev* R, const int4* map) { LGM_BATCH_LOOP(move_body(D, i)) }
__global__ void kb_unclaim(const Dev* R, const int4* map) { LGM_BATCH_LOOP(unclaim_body(D, i)) }
// one block per replica of the list
__global__ void __launch_bounds__(kCompactThreads) kb_compact_inject(const Dev* R, const int* list) {
    __shared__ int warp_sums[32];
    __shared__ double red[32];
    compact_inject_body(R[list[blockIdx.x]], warp_sums, red);
}

// ---- the fused step: one block per replica, every phase inside the block ----------
//
// For replicas small enough that one block carries their whole step, the
// phases above run back to back inside one kernel with __syncthreads between
// them, for many steps per launch.  The phase bodies are the ones the
// separate kernels call, over the same index ranges, with a block-uniform
// loop (every thread runs the same iterations, so the warp-level sums in
// move_body see full warps); __syncthreads orders their global-memory writes
// as the kernel boundaries do.  Only the pair sum differs in form.


// The replica's pair sum inside the block: for every target the arithmetic of
// pair_tile with a single source split -- runs of kSUB sources in FP32 (r^2 - 1/2
// exact, MUFU rsqrt, predicated FFMA), each run folded into FP64 in source
// order, |run sum| added to the FP32 norm -- so the partials equal those of the
// pair kernel with one split bit for bit.  One target per thread at a time:
// every thread reads the same source record at a time (one broadcast load per
// warp, an L1 hit after the first warp).  Carrying 2-4 targets per thread
// through the source loop measured slower here (fewer threads busy, more
// registers).  A charge class is padded to whole chunks with records of
// charge 0; its runs past the class's live charges add exact zeros and are
// skipped.
__device__ void fused_pair_body(const Dev& D) {
    const int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
    const int nd = D.dq != 0 ? D.nd : 0;
    const int pe = (ne + CH - 1) / CH * CH, ph = (nh + CH - 1) / CH * CH;
    const int start[3] = {0, pe, pe + ph}, count[3] = {ne, nh, nd};
    const int t = 2 * (ne + nh);
    const int tpad = D.cnt[I_TPAD];
    const float4* geo = D.geo;
    const float2* qq = D.qq;
    const float* gtab = D.gtab;
    const int gtab_k = D.gtab_k, gauss = D.gauss;
    const unsigned ulim = __float_as_uint((float)D.cutoff2 - 0.5f);
    for (int g = threadIdx.x; g < D.nterms * t; g += blockDim.x) {
        const int slot = g / t;
        const int p = slot * tpad + (g - slot * t);
        const float4 tg = D.tgt[p];
        double acc64 = 0.0;
        float nrm = 0.f;
        for (int c = 0; c < 3; ++c) {
            const int s1 = start[c] + count[c];
            for (int r0 = start[c]; r0 < s1; r0 += kSUB) {
                const int r1 = min(r0 + kSUB, s1);
                float acc = 0.f;
                for (int j = r0; j < r1; ++j) {
                    const float4 g0 = geo[2 * j], g1 = geo[2 * j + 1];
                    float u = __fadd_rn(g1.z, tg.w);  // d + |t|^2
                    u = __fmaf_rn(tg.x, g0.x, u);
                    u = __fmaf_rn(tg.y, g0.z, u);
                    u = __fmaf_rn(tg.z, g1.x, u);     // r^2 - 1/2, exact
                    const float r2 = __fadd_rn(u, 0.5f);
                    float w = rsqrt_mufu(r2);
                    if (gauss) {
                        const int ix = min(__float_as_int(r2 + 8388608.f) & 0x7fffff, gtab_k);
                        w = fminf(gtab[ix], w);
                    }
                    fma_if_below(acc, qq[j].x, w, __float_as_uint(u), ulim);
                }
                acc64 += (double)acc;
                nrm += fabsf(acc);
            }
        }
        D.part[p] = acc64;
        D.part_norm[p] = nrm;
    }
}

#define LGM_BLOCK_LOOP(BOUND, CALL)                                                     \
    for (int base_ = 0; base_ < (BOUND); base_ += (int)blockDim.x) {                  \
        const int i = base_ + (int)threadIdx.x;                                       \
        CALL;                                                                         \
    }

// Block b advances replica list[b] by `steps` steps.  `recomb` is the batch's
// flag (the recombination phases run for every replica of a batch in which any
// replica recombines, as the separate kernels do).  The replica's descriptor
// is copied to shared memory once; each phase loops over the live charges
// counted at the phase's start, not over the capacity.
template <int NT>
__global__ void __launch_bounds__(NT) kb_fused(const Dev* R, const int* list, int steps, int recomb) {
    __shared__ double2 red[NT];
    __shared__ int warp_sums[32];
    __shared__ Dev sD;
    {
        static_assert(sizeof(Dev) % 4 == 0, "word copy");
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&R[list[blockIdx.x]]);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sD);
        for (int w = threadIdx.x; w < (int)(sizeof(Dev) / 4); w += NT) dst[w] = src[w];
    }
    __syncthreads();
    const Dev& D = sD;
    const int nd = D.dq != 0 ? D.nd : 0;
    for (int s = 0; s < steps; ++s) {
        int ne = D.cnt[I_NE], nh = D.cnt[I_NH];
        LGM_BLOCK_LOOP(max(1, ne + nh), choose_body(D, i))
        __syncthreads();
        if (D.coulomb) {
            const int nsrc = (ne + CH - 1) / CH * CH + (nh + CH - 1) / CH * CH +
                             (nd + CH - 1) / CH * CH;
            const int tpad = (2 * (ne + nh) + 63) / 64 * 64;
            LGM_BLOCK_LOOP(max(nsrc, tpad), pack_body(D, i))
            __syncthreads();
            fused_pair_body(D);
            __syncthreads();
            LGM_BLOCK_LOOP(2 * (ne + nh), finalize_body(D, i))
            __syncthreads();
        }
        LGM_BLOCK_LOOP(ne + nh, decide_body(D, i))
        __syncthreads();
        if (D.coulomb) {
            guard_body(D, 0, 1, red);
            __syncthreads();
        }
        if (recomb) {
            LGM_BLOCK_LOOP(nh, hmap_body(D, i, true))
            __syncthreads();
            LGM_BLOCK_LOOP(ne, recomb_propose_body(D, i))
            __syncthreads();
            LGM_BLOCK_LOOP(ne, recomb_resolve_body(D, i))
            __syncthreads();
            LGM_BLOCK_LOOP(max(ne, nh), recomb_reset_body(D, i))
            __syncthreads();
        }
        LGM_BLOCK_LOOP(ne + nh, claim_body(D, i))
        __syncthreads();
        LGM_BLOCK_LOOP(ne + nh, move_body(D, i))
        __syncthreads();
        LGM_BLOCK_LOOP(ne + nh, unclaim_body(D, i))
        __syncthreads();
        compact_inject_body(D, warp_sums, reinterpret_cast<double*>(red));
        __syncthreads();
    }
}
// Block sizes of the fused step: small replicas fill 128 threads, larger 256.
constexpr int kFusedSmallCharges = 512;

// ---- host side -------------------------------------------------------------------

struct Stream {
    uint32_t seed, replica, purpose;
    uint32_t next = 0;
    Philox4 draw() { return philox4x32_10(next++, 0u, purpose, 0u, seed, replica); }
    uint32_t below(uint32_t n) { return uint_below(draw().w[0], n); }
    // Box-Muller (the reference draws boost::normal_distribution, rand.cpp:61-66)
    double normal(double mean, double sigma) {
        const Philox4 r = draw();
        const double u1 = (unit_double(r.w[0], r.w[1]) * 9007199254740991.0 + 1.0) / 9007199254740992.0;
        const double u2 = unit_double(r.w[2], r.w[3]);
        return mean + sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
};

void host_neighbors1(int X, int Y, int Z, int site, std::vector<int>& nb) {
    nb.clear();
    const int XY = X * Y;
    const int z = site / XY, y = site / X - z * Y, x = site % X;
    auto S = [&](int a, int b, int c) { nb.push_back(X * (b + c * Y) + a); };
    if (x > 0) S(x - 1, y, z);
    if (x < X - 1) S(x + 1, y, z);
    if (y > 0) S(x, y - 1, z);
    if (y < Y - 1) S(x, y + 1, z);
    if (z > 0) S(x, y, z - 1);
    if (z < Z - 1) S(x, y, z + 1);
    const int V = X * Y * Z;
    if (x == 0) nb.push_back(V + E_DRAIN_L);  // electron grid drains (cubicgrid.cpp:447-468)
    if (x == X - 1) nb.push_back(V + E_DRAIN_R);
}

}  // namespace

// Bump allocator over large device chunks, owned by a batch: its replicas take
// their buffers from it instead of one cudaMalloc each, and the chunks are
// freed together when the batch is destroyed.
struct DevicePool {
    std::vector<void*> chunks;
    char* cur = nullptr;
    size_t left = 0;
    cudaError_t take(size_t bytes, void** out) {
        bytes = (bytes + 255) / 256 * 256;
        if (bytes > left) {
            const size_t sz = std::max(bytes, (size_t)256 << 20);
            char* c = nullptr;
            const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&c), sz);
            if (e != cudaSuccess) return e;
            chunks.push_back(c);
            cur = c;
            left = sz;
        }
        *out = cur;
        cur += bytes;
        left -= bytes;
        return cudaSuccess;
    }
    void release() {
        for (void* c : chunks) cudaFree(c);
        chunks.clear();
        cur = nullptr;
        left = 0;
    }
};

struct lgm_kmc {
    lgm_params p{};
    DevicePool* pool = nullptr;  // a batch's pool, or null: own allocations
    bool own_stream = true;
    const lgm_world_config* wcfg = nullptr;  // checkpointed world (creation only)
    std::vector<unsigned long long> flux0;   // restored flux counters (our layout)
    int device = 0;
    uint32_t replica = 0;
    int V = 0, max_e = 0, max_h = 0;
    std::vector<double> pot;
    std::vector<int32_t> defects, traps, e0, h0;
    std::vector<double> trap_pots;
    Dev D{};
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<void*> allocs;
    float* gtab = nullptr;
    int gtab_k = 0;
    int pair_blocks = 0, pair_tiles = 0;
    int cull_grid = 0;  // persistent grid of the culled pair kernel (one wave)
    int cull_tiles = 0; // target tiles of the culled pair sum (kCTile targets each)
    bool cull_ok = false;  // the culled pair sum's buffers exist
    int sm_count = 0;   // SMs of the device (the guard's grid)
    std::string err;
};

namespace {

thread_local std::string g_kmc_create_error;

lgm_status kfail(lgm_kmc* k, lgm_status s, const std::string& m) {
    if (k) k->err = m;
    return s;
}

#define KCUDA(k, call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return kfail((k), LGM_ERR_CUDA, std::string(#call ": ") + \
                                                               cudaGetErrorString(e_));  \
    } while (0)

template <class T>
lgm_status dalloc(lgm_kmc* k, T** p, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    if (k->pool) {
        KCUDA(k, k->pool->take(bytes, reinterpret_cast<void**>(p)));
        return LGM_OK;
    }
    KCUDA(k, cudaMalloc(reinterpret_cast<void**>(p), bytes));
    k->allocs.push_back(*p);
    return LGM_OK;
}

// Slices of one device allocation: add() records where each pointer goes and
// its size, commit() makes one cudaMalloc and hands out 256-byte aligned slices.
struct Arena {
    std::vector<std::pair<void**, size_t>> slots;
    template <typename T>
    void add(T** p, size_t n) {
        slots.emplace_back(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
    }
    lgm_status commit(lgm_kmc* k) {
        size_t total = 0;
        for (auto& s : slots) total += (s.second + 255) / 256 * 256;
        char* base = nullptr;
        if (k->pool) {
            KCUDA(k, k->pool->take(std::max<size_t>(total, 256), reinterpret_cast<void**>(&base)));
        } else {
            KCUDA(k, cudaMalloc(reinterpret_cast<void**>(&base), std::max<size_t>(total, 256)));
            k->allocs.push_back(base);
        }
        size_t off = 0;
        for (auto& s : slots) {
            *s.first = base + off;
            off += (s.second + 255) / 256 * 256;
        }
        return LGM_OK;
    }
};

// World::initialize (world.cpp:589-650) on one Philox stream: every set-up
// draw comes from the sequential counter {n, 0, RNG_SETUP, 0} in the order the
// reference consumes its generator -- placeDefects, placeElectrons,
// placeHoles, then setPotentialTraps (seeds, growth, the Gaussian spread) --
// so the reference's own set-up code, given the same draws, builds the same
// world.  The site.disorder extension draws from its own stream afterwards.
lgm_status build_world(lgm_kmc* k) {
    const lgm_params& p = k->p;
    const int X = p.grid_x, Y = p.grid_y, Z = p.grid_z, V = X * Y * Z;
    k->V = V;
    const uint32_t seed = (uint32_t)(p.random_seed & 0xffffffffu);
    k->max_e = (int)(p.electron_percentage * (double)V);
    k->max_h = (int)(p.hole_percentage * (double)V);
    const int max_d = (int)(p.defect_percentage * (double)V);
    const int max_t = (int)(p.trap_percentage * (double)V);
    std::vector<uint8_t> is_def(V, 0), is_trap(V, 0);
    const lgm_world_config* w = k->wcfg;
    Stream r{seed, k->replica, RNG_SETUP + 0};
    // placeDefects (world.cpp:659-757): listed defects first, the rest drawn
    {
        const int given = w ? w->n_defects : 0;
        if (given < 0 || given > max_d || (given && !w->defects))
            return kfail(k, LGM_ERR_INVALID_ARGUMENT, "langmuir: invalid number of defects in checkpoint");
        for (int i = 0; i < given; ++i) {
            const int s = w->defects[i];
            if (s < 0 || s >= V) return kfail(k, LGM_ERR_OUT_OF_RANGE, "defect site out of range");
            if (is_def[s]) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "langmuir: defect already exists");
            is_def[s] = 1;
            k->defects.push_back(s);
        }
        long tries = 0;
        while ((int)k->defects.size() < max_d) {
            if (++tries > 10L * V) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "can not seed defects");
            const int s = (int)r.below((uint32_t)V);
            if (!is_def[s]) { is_def[s] = 1; k->defects.push_back(s); }
        }
    }
    // placeElectrons / placeHoles (world.cpp:759-959): listed sites first, then
    // SourceAgent::tryToSeed at uniform sites (sourceagent.cpp:71-80,
    // validToInject 192-232) up to max * seed.charges
    auto seed_carriers = [&](int max, std::vector<int32_t>& out) -> bool {
        std::vector<uint8_t> occ(V, 0);
        for (int s : out) occ[s] = 1;
        long tries = 0;
        for (int i = (int)out.size(); i < max * p.seed_charges;) {
            if (++tries > 10L * V) return false;
            const int s = (int)r.below((uint32_t)V);
            if (!occ[s] && !is_def[s] && (int)out.size() < max) {
                occ[s] = 1;
                out.push_back(s);
                ++i;
            }
        }
        return true;
    };
    auto given = [&](const int32_t* ids, int n, int max, std::vector<int32_t>& out,
                     const char* what) -> lgm_status {
        if (n < 0 || n > max || (n && !ids))
            return kfail(k, LGM_ERR_INVALID_ARGUMENT,
                         std::string("langmuir: invalid number of ") + what + " in checkpoint");
        std::vector<uint8_t> occ(V, 0);
        for (int i = 0; i < n; ++i) {
            const int s = ids[i];
            if (s < 0 || s >= V || occ[s] || is_def[s])
                return kfail(k, LGM_ERR_INVALID_ARGUMENT, std::string("langmuir: can not inject ") +
                                                              what + " at site " + std::to_string(s));
            occ[s] = 1;
            out.push_back(s);
        }
        return LGM_OK;
    };
    if (w) {
        lgm_status st;
        if ((st = given(w->electrons, w->n_electrons, k->max_e, k->e0, "electron")) != LGM_OK) return st;
        if ((st = given(w->holes, w->n_holes, k->max_h, k->h0, "hole")) != LGM_OK) return st;
        // World::setFluxInfo (world.cpp:1189-1318) into this library's counter layout:
        // eSL eSR hSL hSR (0-7), eDL eDR hDL hDR (8-15), exciton source (16-17),
        // recombination (18-19), each (attempts, successes)
        if (w->n_flux) {
            if (!w->flux) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "flux state without values");
            const uint64_t* f = w->flux;
            k->flux0.assign(20, 0ull);
            auto put = [&](int agent, int at) { k->flux0[2 * agent] = f[at]; k->flux0[2 * agent + 1] = f[at + 1]; };
            const bool solar = std::string(p.simulation_type) == "solarcell";
            if (w->n_flux == 4 && !solar) {
                put(0, 0); put(5, 2);
            } else if ((w->n_flux == 10 || w->n_flux == 12) && solar) {
                put(8, 0); put(4, 2); put(6, 4); put(5, 6); put(7, 8);
                if (w->n_flux == 12) put(9, 10);
            } else if (w->n_flux == 20) {
                put(0, 0); put(1, 2); put(2, 4); put(3, 6); put(8, 8);
                put(4, 10); put(5, 12); put(6, 14); put(7, 16); put(9, 18);
            } else {
                return kfail(k, LGM_ERR_PARSE, "langmuir: do not recognize [FluxInfo] format (of size " +
                                                   std::to_string(w->n_flux) + ")");
            }
        }
    }
    if (!seed_carriers(k->max_e, k->e0))
        return kfail(k, LGM_ERR_INVALID_ARGUMENT, "can not seed electrons");
    if (!seed_carriers(k->max_h, k->h0))
        return kfail(k, LGM_ERR_INVALID_ARGUMENT, "can not seed holes");
    // setPotentialTraps (potential.cpp:74-244): listed traps first (with their
    // potentials or trap.potential), then random seeds and growth onto
    // neighbours of the random ones; the Gaussian spread applies to those only
    {
        const int forced = w ? w->n_traps : 0;
        if (forced < 0 || forced > max_t || (forced && !w->traps))
            return kfail(k, LGM_ERR_INVALID_ARGUMENT, "langmuir: invalid trap parameters");
        if (forced > 0 && w->n_trap_potentials != 0 &&
            (w->n_trap_potentials != forced || !w->trap_potentials))
            return kfail(k, LGM_ERR_INVALID_ARGUMENT,
                         "langmuir: trapPotential and trap arrays different sizes in checkpoint file");
        for (int i = 0; i < forced; ++i) {
            const int s = w->traps[i];
            if (s < 0 || s >= V) return kfail(k, LGM_ERR_OUT_OF_RANGE, "trap site out of range");
            is_trap[s] = 1;
            k->traps.push_back(s);
            k->trap_pots.push_back(w->n_trap_potentials ? w->trap_potentials[i] : p.trap_potential);
        }
        const int random = max_t - forced;
        int seeds = (int)(random * p.seed_percentage);
        int grown = random - seeds;
        if (random <= 0) { seeds = 0; grown = 0; }
        if (seeds == 0 && grown > 0) { seeds = grown; grown = 0; }
        long tries = 0;
        while ((int)k->traps.size() < forced + seeds) {
            if (++tries > 100L * V + 1000) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "can not seed traps");
            const int s = (int)r.below((uint32_t)V);
            if (!is_trap[s]) { is_trap[s] = 1; k->traps.push_back(s); }
        }
        std::vector<int> nb;
        int progress = 0;
        while (progress < grown) {
            if (++tries > 100L * V + 1000) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "can not grow traps");
            const int n_random = (int)k->traps.size() - forced;
            const int seed_site = k->traps[forced + (int)r.below((uint32_t)n_random)];
            host_neighbors1(X, Y, Z, seed_site, nb);
            const int s = nb[r.below((uint32_t)nb.size())];
            if (s < V && !is_trap[s]) { is_trap[s] = 1; k->traps.push_back(s); ++progress; }
        }
        k->trap_pots.resize(k->traps.size(), p.trap_potential);
        if (std::fabs(p.gaussian_stdev) > 0)
            for (size_t i = forced; i < k->trap_pots.size(); ++i)
                k->trap_pots[i] += r.normal(0.0, p.gaussian_stdev);
    }
    // setPotentialZero / Linear / Gate (potential.cpp:17-72), traps, disorder
    k->pot.assign(V, 0.0);
    const double m = (p.voltage_right - p.voltage_left) / (double)X, b = p.voltage_left;
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Y; ++j)
            for (int z = 0; z < Z; ++z) k->pot[X * (j + z * Y) + i] += m * (i + 0.5) + b;
    if (!(Z == 1 || p.slope_z == 0))
        for (int i = 0; i < X; ++i)
            for (int j = 0; j < Y; ++j)
                for (int z = 0; z < Z; ++z) k->pot[X * (j + z * Y) + i] += p.slope_z * (z + 0.5);
    for (size_t i = 0; i < k->traps.size(); ++i) k->pot[k->traps[i]] += k->trap_pots[i];
    if (p.site_disorder > 0) {
        Stream rd{seed, k->replica, RNG_SETUP + 2};
        for (int s = 0; s < V; ++s) k->pot[s] += rd.normal(0.0, p.site_disorder);
    }
    return LGM_OK;
}

lgm_status upload_carriers(lgm_kmc* k, const int32_t* e, int ne, const int32_t* h, int nh) {
    Dev& D = k->D;
    std::vector<uint8_t> et(k->V + kSpecial, T_EMPTY), ht(k->V + kSpecial, T_EMPTY);
    for (int s : k->defects) et[s] = ht[s] = T_DEFECT;
    for (int i = 0; i < ne; ++i) {
        if (e[i] < 0 || e[i] >= k->V || et[e[i]] != T_EMPTY)
            return kfail(k, LGM_ERR_OUT_OF_RANGE, "electron site invalid or occupied");
        et[e[i]] = T_ELECTRON;
    }
    for (int i = 0; i < nh; ++i) {
        if (h[i] < 0 || h[i] >= k->V || ht[h[i]] != T_EMPTY)
            return kfail(k, LGM_ERR_OUT_OF_RANGE, "hole site invalid or occupied");
        ht[h[i]] = T_HOLE;
    }
    const int V = k->V;
    et[V + 0] = et[V + 1] = et[V + 2] = T_SOURCE;
    et[V + 3] = et[V + 4] = et[V + 5] = T_DRAIN;
    ht[V + 0] = ht[V + 1] = T_SOURCE;
    ht[V + 2] = ht[V + 3] = T_DRAIN;
    KCUDA(k, cudaMemcpy(D.et, et.data(), et.size(), cudaMemcpyHostToDevice));
    KCUDA(k, cudaMemcpy(D.ht, ht.data(), ht.size(), cudaMemcpyHostToDevice));
    if (ne) KCUDA(k, cudaMemcpy(D.e_site, e, sizeof(int32_t) * ne, cudaMemcpyHostToDevice));
    if (nh) KCUDA(k, cudaMemcpy(D.h_site, h, sizeof(int32_t) * nh, cudaMemcpyHostToDevice));
    int32_t c[2] = {ne, nh};
    KCUDA(k, cudaMemcpy(D.cnt + I_NE, c, sizeof c, cudaMemcpyHostToDevice));
    return LGM_OK;
}

using KPairFn = void (*)(PairArgs);

using KCulledFn = void (*)(PairArgs, CullArgs);
KCulledFn kmc_pair_culled(int gauss) {
    return gauss ? &pair_kernel_culled_ws<1, 0, kCNW, kCRP, kCSUB, kCStages, kCMinBlocks, true, false, kCVote>
                 : &pair_kernel_culled_ws<0, 0, kCNW, kCRP, kCSUB, kCStages, kCMinBlocks, true, false, kCVote>;
}
size_t kmc_culled_smem(int tab_k) { return ws_smem_bytes(kCStages, tab_k, 4); }

// the culled replicas of a batch (point charges), one persistent launch
constexpr auto kBatchCulled =
    &pair_kernel_culled_ws_list<kCNW, kCRP, kCSUB, kCStages, kCMinBlocks, true, false, kCVote>;

KPairFn kmc_pair(int gauss, int sorted = 1) {
    if (sorted)
        return gauss ? &pair_kernel<1, 0, kNT, kRP, kSUB, true, true>
                     : &pair_kernel<0, 0, kNT, kRP, kSUB, true, true>;
    return gauss ? &pair_kernel<1, 0, kNT, kRP, kSUB, true> : &pair_kernel<0, 0, kNT, kRP, kSUB, true>;
}

// Launches one kernel of the step with programmatic stream serialization:
// it may be scheduled while the kernel ahead of it is running and waits for
// it in pdl_wait() (every k_* kernel and the pair kernels call it first), so
// the launch gaps inside the captured graph overlap the kernel ahead.
template <typename... P, typename... Args>
cudaError_t kl(void (*f)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               Args... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, f, static_cast<P>(args)...);
}

// One step: kernels in order on k->stream (captured into the graph).
lgm_status enqueue_step(lgm_kmc* k) {
    const Dev& D = k->D;
    cudaStream_t st = k->stream;
    const int nc = std::max(1, D.cap_e + D.cap_h);
    const int blk = 256;
    const int g1 = (nc + blk - 1) / blk;
    KCUDA(k, kl(k_choose, g1, blk, 0, st, D));
    if (D.coulomb) {
        if (D.sorted) {
            const int nz = D.culled ? 3 * (D.ncells + 1) : D.ncells + 1;
            const int nb = std::max(2 * nc, nc + (D.dq != 0 ? D.nd : 0));
            KCUDA(k, kl(k_tbins_zero, (nz + blk - 1) / blk, blk, 0, st, D));
            KCUDA(k, kl(k_tbins, (nb + blk - 1) / blk, blk, 0, st, D));
            KCUDA(k, kl(k_tbins_scan, D.culled ? 2 : 1, 1024, 0, st, D));
            KCUDA(k, kl(k_tscatter, (nb + blk - 1) / blk, blk, 0, st, D));
            if (D.culled) KCUDA(k, kl(k_trank, (2 * nc + blk - 1) / blk, blk, 0, st, D));
        }
        const int npack = std::max(D.src_cap, D.tpad_cap);
        KCUDA(k, kl(k_pack, (npack + blk - 1) / blk, blk, 0, st, D));
        const PairArgs A = pair_args(D);
        if (D.culled) {
            KCUDA(k, kl(k_chunk_boxes, D.src_cap / CH, CH, 0, st, D));
            KCUDA(k, kl(k_cull, k->cull_tiles, kCullThreads, 0, st, D));
            KCUDA(k, kl(kmc_pair_culled(D.gauss), k->cull_grid, kCThreads,
                        kmc_culled_smem(A.tab_k), st, A, cull_args(D)));
        } else {
            KCUDA(k, kl(kmc_pair(D.gauss, D.sorted), dim3(k->pair_tiles, D.splits), kNT,
                        pair_smem_bytes(A.tab_k), st, A));
        }
        if (D.culled) KCUDA(k, kl(k_finalize_culled, (2 * nc + 31) / 32, dim3(32, 3), 0, st, D));
        else KCUDA(k, kl(k_finalize, (2 * nc + blk - 1) / blk, blk, 0, st, D));
    }
    KCUDA(k, kl(k_decide, g1, blk, 0, st, D));
    if (D.coulomb) KCUDA(k, kl(k_guard, 2 * k->sm_count, kGuardThreads, 0, st, D));
    if (D.solar && D.rec_rate > 0) {
        KCUDA(k, kl(k_hmap, g1, blk, 0, st, D));
        KCUDA(k, kl(k_recomb_propose, g1, blk, 0, st, D));
        KCUDA(k, kl(k_recomb_resolve, g1, blk, 0, st, D));
        KCUDA(k, kl(k_recomb_reset, g1, blk, 0, st, D));
    }
    KCUDA(k, kl(k_claim, g1, blk, 0, st, D));
    KCUDA(k, kl(k_move, g1, blk, 0, st, D));
    KCUDA(k, kl(k_unclaim, g1, blk, 0, st, D));
    KCUDA(k, kl(k_compact_inject, 1, kCompactThreads, 0, st, D));
    return LGM_OK;
}

}  // namespace

extern "C" {

// One replica.  pool / shared: a batch's device pool and stream (the batch
// synchronises once after creating all replicas), or null for a standalone one.
static lgm_status kmc_create_impl(const lgm_params* pin, int32_t device, uint32_t replica,
                                  lgm_kmc** out, DevicePool* pool, cudaStream_t shared,
                                  const lgm_world_config* wcfg = nullptr) {
    if (!pin || !out) return LGM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    lgm_kmc* k = new (std::nothrow) lgm_kmc();
    if (!k) return LGM_ERR_INVALID_ARGUMENT;
    k->p = *pin;
    k->pool = pool;
    k->wcfg = wcfg;
    k->replica = replica;
    char msg[256] = {0};
    lgm_status s = lgm_params_check(&k->p, msg, sizeof msg);
    auto bail = [&](lgm_status st, const std::string& m) {
        g_kmc_create_error = m;
        lgm_kmc_destroy(k);
        return st;
    };
    g_kmc_create_error.clear();
    if (s != LGM_OK) return bail(s, msg);
    const lgm_params& p = k->p;
    if (p.recombination_range < 0 || p.recombination_range > 2)
        return bail(LGM_ERR_INVALID_ARGUMENT, "langmuir: recombination.range must be 0, 1 or 2");
    const bool solar = std::string(p.simulation_type) == "solarcell";
    if (p.hopping_range < 1) return bail(LGM_ERR_UNSUPPORTED, "hopping.range 0 has no moves");
    const long long L = std::max<long long>({2LL * p.grid_x, p.grid_y, p.grid_z + 1});
    if (6 * L * L >= (1LL << 22)) return bail(LGM_ERR_UNSUPPORTED, "lattice too large");
    if ((s = build_world(k)) != LGM_OK) return bail(s, k->err);
    k->device = device < 0 ? 0 : device;
    if (cudaSetDevice(k->device) != cudaSuccess) return bail(LGM_ERR_NO_DEVICE, "no device");
    // attribute reads, not cudaGetDeviceProperties: a batch creates thousands of replicas
    int cc_major = 0, n_sms = 0;
    if (cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, k->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, k->device) != cudaSuccess ||
        cc_major != 10)
        return bail(LGM_ERR_NO_DEVICE, "device is not sm_100 (B200)");
    if (shared) {
        k->stream = shared;
        k->own_stream = false;
    } else if (cudaStreamCreateWithFlags(&k->stream, cudaStreamNonBlocking) != cudaSuccess) {
        return bail(LGM_ERR_CUDA, "stream");
    }

    Dev& D = k->D;
    D.X = p.grid_x; D.Y = p.grid_y; D.Z = p.grid_z; D.XY = D.X * D.Y; D.V = k->V;
    D.hr = p.hopping_range;
    D.cap_e = k->max_e; D.cap_h = k->max_h;
    D.nd = (int)k->defects.size(); D.dq = p.defects_charge;
    D.seed = (uint32_t)(p.random_seed & 0xffffffffu); D.replica = replica;
    D.beta = p.inverse_kt; D.exciton_binding = p.exciton_binding;
    D.prefactor = p.electrostatic_prefactor;
    D.guard = p.guard_band;
    D.src_metro = p.source_metropolis ? 1 : 0;
    D.src_coulomb = p.source_coulomb ? 1 : 0;
    D.balance = p.balance_charges ? 1 : 0;
    D.volt_l = p.voltage_left;
    D.volt_r = p.voltage_right;
    D.erffactor = p.coulomb_gaussian_sigma > 0 ? 1.0 / (std::sqrt(2.0) * p.coulomb_gaussian_sigma) : 0.0;
    D.gauss = p.coulomb_gaussian_sigma > 0;
    // sI[1][0][0] = prefactor * iR * eR at r = 1 (potential.cpp:311-323)
    D.sI100 = p.electrostatic_prefactor * (D.gauss ? std::erf(D.erffactor * 1.0) : 1.0);
    // coupling (potential.cpp:326-349)
    {
        const int h = D.hr + 1;
        for (int dx = 0; dx < h; ++dx)
            for (int dy = 0; dy < h; ++dy)
                for (int dz = 0; dz < h; ++dz) {
                    const double r = std::sqrt((double)(dx * dx + dy * dy + dz * dz));
                    D.coupling[(dx * h + dy) * h + dz] =
                        (1.0 / 3.0) * std::pow(3.0, r - 1) * std::pow(1.0 / 27.0, r - 1);
                }
        D.coupling[0] = 0.0;
    }
    // World::createSources/createDrains rates (world.cpp:982-1030, 1110-1150)
    auto smart = [](double r, double dflt) { return r < 0 ? dflt : r; };
    D.solar = solar;
    if (!solar) {
        D.rate_src[0] = smart(p.e_source_l_rate, p.source_rate);
        D.rate_src[1] = smart(p.e_source_r_rate, 0.0);
        D.rate_src[2] = smart(p.h_source_l_rate, 0.0);
        D.rate_src[3] = smart(p.h_source_r_rate, 0.0);
        D.rate_drain[0] = smart(p.e_drain_l_rate, 0.0);
        D.rate_drain[1] = smart(p.e_drain_r_rate, p.drain_rate);
        D.rate_drain[2] = smart(p.h_drain_l_rate, 0.0);
        D.rate_drain[3] = smart(p.h_drain_r_rate, 0.0);
        D.gen_rate = 0.0;
        D.rec_rate = 0.0;
    } else {
        D.rate_src[0] = smart(p.e_source_l_rate, 0.0);
        D.rate_src[1] = smart(p.e_source_r_rate, 0.0);
        D.rate_src[2] = smart(p.h_source_l_rate, 0.0);
        D.rate_src[3] = smart(p.h_source_r_rate, 0.0);
        D.rate_drain[0] = smart(p.e_drain_l_rate, p.drain_rate);
        D.rate_drain[1] = smart(p.e_drain_r_rate, p.drain_rate);
        D.rate_drain[2] = smart(p.h_drain_l_rate, p.drain_rate);
        D.rate_drain[3] = smart(p.h_drain_r_rate, p.drain_rate);
        D.gen_rate = smart(p.generation_rate, p.source_rate);
        const double area = (double)p.grid_x * p.grid_y;
        if (p.source_scale_area > 0 && p.source_scale_area != area)
            D.gen_rate *= area / p.source_scale_area;
        D.rec_rate = p.recombination_rate;
    }
    D.rec_range = p.recombination_range;
    D.confine = p.morphology_confine;
    D.gen_iface = p.generation_interface;
    // createSources / createDrains sanity checks (world.cpp:1032-1068, 1158-1186)
    if (D.rate_src[0] == 0 && D.rate_src[1] == 0 && D.rate_src[2] == 0 && D.rate_src[3] == 0 &&
        D.gen_rate == 0)
        return bail(LGM_ERR_INVALID_ARGUMENT, "langmuir: all sources have zero rate");
    if (k->max_e == 0 && (D.rate_src[0] > 0 || D.rate_src[1] > 0))
        return bail(LGM_ERR_INVALID_ARGUMENT,
                    "langmuir: an electron source rate > 0, yet maxElectronAgents() == 0");
    if (k->max_h == 0 && (D.rate_src[2] > 0 || D.rate_src[3] > 0))
        return bail(LGM_ERR_INVALID_ARGUMENT,
                    "langmuir: a hole source rate > 0, yet maxHoleAgents() == 0");
    if (k->max_e == 0 && D.gen_rate > 0)
        return bail(LGM_ERR_INVALID_ARGUMENT,
                    "langmuir: generation.rate > 0, yet maxElectronAgents() == 0");
    if (D.rate_drain[0] == 0 && D.rate_drain[1] == 0 && D.rate_drain[2] == 0 &&
        D.rate_drain[3] == 0 && D.rec_rate == 0)
        return bail(LGM_ERR_INVALID_ARGUMENT, "langmuir: all drains have zero rate");
    if (k->max_e > 0 && D.rate_drain[0] <= 0 && D.rate_drain[1] <= 0 && D.rec_rate <= 0)
        return bail(LGM_ERR_INVALID_ARGUMENT,
                    "langmuir: all electron drain rates are zero, yet maxElectronAgents() > 0");
    if (k->max_h > 0 && D.rate_drain[2] <= 0 && D.rate_drain[3] <= 0 && D.rec_rate <= 0)
        return bail(LGM_ERR_INVALID_ARGUMENT,
                    "langmuir: all hole drain rates are zero, yet maxHoleAgents() > 0");
    D.coulomb = p.coulomb_carriers;
    D.terms = LGM_TERM_DIRECT | ((p.image_charges & 1) ? LGM_TERM_IMAGE_LEFT : 0u) |
              ((p.image_charges & 2) ? LGM_TERM_IMAGE_RIGHT : 0u);
    D.nterms = 1 + ((p.image_charges & 1) ? 1 : 0) + ((p.image_charges & 2) ? 1 : 0);
    D.cutoff2 = p.electrostatic_cutoff * p.electrostatic_cutoff;

    const int ncap = std::max(1, D.cap_e + D.cap_h);
    const int nd_src = D.dq != 0 ? D.nd : 0;
    D.src_cap = ((D.cap_e + CH - 1) / CH + (D.cap_h + CH - 1) / CH + (nd_src + CH - 1) / CH) * CH;
    D.src_cap = std::max(D.src_cap, CH);
    D.tpad_cap = (2 * ncap + 63) / 64 * 64;
    const int tphys_cap = D.nterms * D.tpad_cap;
    k->pair_tiles = (tphys_cap + kTile - 1) / kTile;
    int bps = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kmc_pair(D.gauss), kNT, pair_smem_bytes(64));
    // three waves of resident CTAs, as for the single pair sums (lgm_api.cu)
    k->sm_count = n_sms;
    D.splits = std::max(1, std::min({64, 3 * n_sms * std::max(1, bps) / k->pair_tiles,
                                     D.src_cap / CH}));
    lgm_status st;
    // every buffer of the replica in one allocation (256-byte aligned slices)
    Arena arena;
#define DA(ptr, n) arena.add(&(ptr), (size_t)(n))
    DA(D.pot, k->V);
    DA(D.et, k->V + kSpecial);
    DA(D.ht, k->V + kSpecial);
    DA(D.e_site, std::max(D.cap_e, 1)); DA(D.h_site, std::max(D.cap_h, 1));
    DA(D.e_f, std::max(D.cap_e, 1)); DA(D.h_f, std::max(D.cap_h, 1));
    DA(D.defects, std::max(D.nd, 1));
    DA(D.claim_e, k->V); DA(D.claim_h, k->V);
    DA(D.outcome, ncap); DA(D.de, ncap); DA(D.accept, ncap); DA(D.flagged, ncap);
    DA(D.gpart, (size_t)ncap * kGuardSplits); DA(D.gdone, ncap);
    DA(D.cnt, I_NUM); DA(D.ctr, C_NUM);
    DA(D.geo, 2 * D.src_cap); DA(D.qq, D.src_cap);
    DA(D.tgt, tphys_cap + kTile);
    // The pair sum culls source chunks beyond the cutoff when the replica has
    // room for kCullMinChunks of them: a standalone replica always, a batch's
    // replica when the batch puts it on the per-phase kernels (partition_batch
    // sets D.culled; its partials then take either layout).
    const int src_chunks = D.src_cap / CH;
    k->cull_ok = D.coulomb && src_chunks >= kCullMinChunks;
    D.culled = (k->cull_ok && !pool) ? 1 : 0;
    k->cull_tiles = (tphys_cap + kCTile - 1) / kCTile;
    D.max_items = std::min(kMaxItemsPerTile, (src_chunks + kCullPerItem - 1) / kCullPerItem);
    const size_t part_cull = (size_t)k->cull_tiles * D.max_items * kCTile;
    const size_t part_n = D.culled ? part_cull
                          : k->cull_ok ? std::max(part_cull, (size_t)D.splits * tphys_cap)
                                       : (size_t)D.splits * tphys_cap;
    DA(D.part, part_n); DA(D.part_norm, part_n);
    if (k->cull_ok) {
        DA(D.skey, D.cap_e + D.cap_h + nd_src); DA(D.stmp, D.cap_e + D.cap_h + nd_src);
        DA(D.ttmp, 2 * ncap);
        DA(D.cbox, src_chunks); DA(D.gbox, (size_t)src_chunks * kGroupsPerChunk);
        DA(D.live, (size_t)k->cull_tiles * src_chunks);
        DA(D.items, (size_t)k->cull_tiles * D.max_items);
        DA(D.item_count, 3); DA(D.tile_first, k->cull_tiles); DA(D.tile_items, k->cull_tiles);
        DA(D.chist, kCostBuckets); DA(D.corder, (size_t)k->cull_tiles * D.max_items);
    }
    DA(D.Vt, 2 * ncap); DA(D.Nt, 2 * ncap);
    DA(D.err, 1);
    DA(D.phase, k->V);
    DA(D.bonds, (D.gen_iface ? 12 * (size_t)k->V : 2));
    DA(D.h_at, k->V);
    DA(D.rclaim, std::max(D.cap_h, 1));
    DA(D.e_rch, std::max(D.cap_e, 1));
    DA(D.e_rm, std::max(D.cap_e, 1));
    DA(D.h_rm, std::max(D.cap_h, 1));
    DA(D.w64, std::max(D.cutoff2, 1));
    const std::vector<int32_t> crank =
        cell_ranks(p.grid_x, p.grid_y, p.grid_z, &D.cell_shift, &D.cells_x, &D.cells_y);
    D.ncells = (int)crank.size();
    D.sorted = D.coulomb ? 1 : 0;
    int32_t* crank_d = nullptr;
    DA(crank_d, D.ncells);
    DA(D.bins, D.ncells + 2);
    if (k->cull_ok) DA(D.sbins, 3 * (D.ncells + 1) + 1);
    DA(D.tkey, 2 * ncap);
    DA(D.tperm, 2 * ncap);
#undef DA
    if ((st = arena.commit(k)) != LGM_OK) return bail(st, k->err);
    if (D.gauss) {
        // erf(f sqrt(k))/sqrt(k) where it differs from 1/sqrt(k) in FP32; NaN past it
        const int c2 = D.cutoff2;
        int kmax = 1;
        while (kmax < c2 && std::erfc(D.erffactor * std::sqrt((double)kmax)) >= 0x1p-30) ++kmax;
        std::vector<float> gt(kmax + 1, 0.f);
        for (int i = 1; i < kmax; ++i) {
            const double r = std::sqrt((double)i);
            gt[i] = (float)(std::erf(D.erffactor * r) / r);
        }
        gt[kmax] = std::nanf("");
        k->gtab_k = kmax;
        if ((st = dalloc(k, &k->gtab, gt.size())) != LGM_OK) return bail(st, k->err);
        if (cudaMemcpy(k->gtab, gt.data(), gt.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(LGM_ERR_CUDA, "table upload");
        D.gtab = k->gtab;
        D.gtab_k = kmax;
        for (int sorted = 0; sorted < 2; ++sorted)
            cudaFuncSetAttribute(kmc_pair(1, sorted), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pair_smem_bytes(kmax));
        cudaFuncSetAttribute(kmc_pair_culled(1), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kmc_culled_smem(kmax));
    }
    cudaMemcpy(crank_d, crank.data(), sizeof(int32_t) * crank.size(), cudaMemcpyHostToDevice);
    D.cell_rank = crank_d;
    if (D.culled) {
        int cbps = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cbps, kmc_pair_culled(D.gauss), kCThreads,
                                                      kmc_culled_smem(D.gauss ? D.gtab_k : 0));
        k->cull_grid = n_sms * std::max(1, cbps);
    }
    {
        std::vector<double> w(std::max(D.cutoff2, 1), 0.0);
        for (int r2 = 1; r2 < D.cutoff2; ++r2) {
            const double r = std::sqrt((double)r2);
            w[r2] = D.gauss ? std::erf(D.erffactor * r) / r : 1.0 / r;
        }
        cudaMemcpy(D.w64, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice);
    }
    cudaMemcpy(D.pot, k->pot.data(), sizeof(double) * k->V, cudaMemcpyHostToDevice);
    if (D.nd) cudaMemcpy(D.defects, k->defects.data(), sizeof(int32_t) * D.nd, cudaMemcpyHostToDevice);
    std::vector<int32_t> claims(k->V, INT_MAX);
    cudaMemcpy(D.claim_e, claims.data(), sizeof(int32_t) * k->V, cudaMemcpyHostToDevice);
    cudaMemcpy(D.claim_h, claims.data(), sizeof(int32_t) * k->V, cudaMemcpyHostToDevice);
    cudaMemcpy(D.rclaim, claims.data(), sizeof(int32_t) * std::max(D.cap_h, 1), cudaMemcpyHostToDevice);
    cudaMemset(D.h_at, 0xff, sizeof(int32_t) * k->V);  // -1
    cudaMemset(D.phase, 0, k->V);
    cudaMemset(D.e_rm, 0, std::max(D.cap_e, 1));
    cudaMemset(D.h_rm, 0, std::max(D.cap_h, 1));
    cudaMemset(D.cnt, 0, sizeof(int32_t) * I_NUM);
    cudaMemset(D.gdone, 0, sizeof(int32_t) * ncap);
    cudaMemset(D.ctr, 0, sizeof(unsigned long long) * C_NUM);
    if (!k->flux0.empty())
        cudaMemcpy(D.ctr, k->flux0.data(), sizeof(unsigned long long) * k->flux0.size(),
                   cudaMemcpyHostToDevice);
    cudaMemset(D.err, 0, sizeof(unsigned));
    int32_t step0 = (int32_t)p.current_step;
    cudaMemcpy(D.cnt + I_STEP, &step0, sizeof step0, cudaMemcpyHostToDevice);
    if ((st = upload_carriers(k, k->e0.data(), (int)k->e0.size(), k->h0.data(),
                              (int)k->h0.size())) != LGM_OK)
        return bail(st, k->err);
    if (!pool && cudaDeviceSynchronize() != cudaSuccess) return bail(LGM_ERR_CUDA, "set-up");
    k->wcfg = nullptr;  // the caller's arrays are not kept
    *out = k;
    return LGM_OK;
}

lgm_status lgm_kmc_create(const lgm_params* pin, int32_t device, uint32_t replica, lgm_kmc** out) {
    return kmc_create_impl(pin, device, replica, out, nullptr, nullptr);
}

lgm_status lgm_kmc_create_from(const lgm_params* pin, const lgm_world_config* w, int32_t device,
                               uint32_t replica, lgm_kmc** out) {
    if (!w) return LGM_ERR_INVALID_ARGUMENT;
    return kmc_create_impl(pin, device, replica, out, nullptr, nullptr, w);
}

lgm_status lgm_kmc_world_host(const lgm_params* pin, uint32_t replica, double* site_energy,
                              int32_t* defects, int32_t d_cap, int32_t* traps, double* trap_pots,
                              int32_t t_cap, int32_t* electrons, int32_t e_cap, int32_t* holes,
                              int32_t h_cap, int32_t* counts) {
    if (!pin || !counts) return LGM_ERR_INVALID_ARGUMENT;
    lgm_kmc k;
    k.p = *pin;
    k.replica = replica;
    char msg[256] = {0};
    lgm_status st = lgm_params_check(&k.p, msg, sizeof msg);
    if (st != LGM_OK) {
        g_kmc_create_error = msg;
        return st;
    }
    if ((st = build_world(&k)) != LGM_OK) {
        g_kmc_create_error = k.err;
        return st;
    }
    counts[0] = (int32_t)k.defects.size();
    counts[1] = (int32_t)k.traps.size();
    counts[2] = (int32_t)k.e0.size();
    counts[3] = (int32_t)k.h0.size();
    if (counts[0] > d_cap || counts[1] > t_cap || counts[2] > e_cap || counts[3] > h_cap)
        return LGM_ERR_CAPACITY;
    if (site_energy) std::memcpy(site_energy, k.pot.data(), sizeof(double) * k.pot.size());
    if (defects) std::memcpy(defects, k.defects.data(), sizeof(int32_t) * k.defects.size());
    if (traps) std::memcpy(traps, k.traps.data(), sizeof(int32_t) * k.traps.size());
    if (trap_pots) std::memcpy(trap_pots, k.trap_pots.data(), sizeof(double) * k.trap_pots.size());
    if (electrons) std::memcpy(electrons, k.e0.data(), sizeof(int32_t) * k.e0.size());
    if (holes) std::memcpy(holes, k.h0.data(), sizeof(int32_t) * k.h0.size());
    return LGM_OK;
}

lgm_status lgm_kmc_destroy(lgm_kmc* k) {
    if (!k) return LGM_OK;
    cudaSetDevice(k->device);
    if (k->stream && k->own_stream) cudaStreamSynchronize(k->stream);
    if (k->exec) cudaGraphExecDestroy(k->exec);
    if (k->graph) cudaGraphDestroy(k->graph);
    for (void* p : k->allocs) cudaFree(p);
    if (k->stream && k->own_stream) cudaStreamDestroy(k->stream);
    delete k;
    return LGM_OK;
}

const char* lgm_kmc_last_error(const lgm_kmc* k) {
    return k ? k->err.c_str() : g_kmc_create_error.c_str();
}

lgm_status lgm_kmc_run(lgm_kmc* k, int32_t steps) {
    if (!k || steps < 0) return LGM_ERR_INVALID_ARGUMENT;
    KCUDA(k, cudaSetDevice(k->device));
    if (!k->exec && steps > 0) {
        KCUDA(k, cudaStreamBeginCapture(k->stream, cudaStreamCaptureModeThreadLocal));
        lgm_status s = enqueue_step(k);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(k->stream, &g);
        if (s != LGM_OK) { if (g) cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) return kfail(k, LGM_ERR_CUDA, "graph capture failed");
        k->graph = g;
        KCUDA(k, cudaGraphInstantiate(&k->exec, g, 0));
    }
    for (int i = 0; i < steps; ++i) KCUDA(k, cudaGraphLaunch(k->exec, k->stream));
    KCUDA(k, cudaStreamSynchronize(k->stream));
    unsigned e = 0;
    KCUDA(k, cudaMemcpy(&e, k->D.err, sizeof e, cudaMemcpyDeviceToHost));
    if (e & DEVERR_TIMEOUT) return kfail(k, LGM_ERR_TIMEOUT, "a bounded device wait ran out");
    if (e & DEVERR_STATE)
        return kfail(k, LGM_ERR_STATE,
                     "langmuir: can not balance the charges (balance.charges, 1024 tries)");
    if (e) return kfail(k, LGM_ERR_STATE, "device reported an error during the step");
    return LGM_OK;
}

lgm_status lgm_kmc_stats_get(lgm_kmc* k, lgm_kmc_stats* s) {
    if (!k || !s) return LGM_ERR_INVALID_ARGUMENT;
    KCUDA(k, cudaSetDevice(k->device));
    KCUDA(k, cudaStreamSynchronize(k->stream));
    int32_t c[I_NUM];
    unsigned long long ctr[C_NUM];
    KCUDA(k, cudaMemcpy(c, k->D.cnt, sizeof c, cudaMemcpyDeviceToHost));
    KCUDA(k, cudaMemcpy(ctr, k->D.ctr, sizeof ctr, cudaMemcpyDeviceToHost));
    std::memset(s, 0, sizeof *s);
    s->step = (uint32_t)c[I_STEP];
    s->electrons = c[I_NE];
    s->holes = c[I_NH];
    s->max_electrons = k->max_e;
    s->max_holes = k->max_h;
    s->defects = (int32_t)k->defects.size();
    s->traps = (int32_t)k->traps.size();
    s->proposals = ctr[C_PROPOSALS];
    s->accepted = ctr[C_ACCEPTED];
    s->guard_evaluations = ctr[C_GUARD];
    for (int i = 0; i < 20; ++i) s->counters[i] = ctr[i];
    return LGM_OK;
}

lgm_status lgm_kmc_get_carriers(lgm_kmc* k, int32_t* e, int32_t e_cap, int32_t* h, int32_t h_cap) {
    if (!k) return LGM_ERR_INVALID_ARGUMENT;
    KCUDA(k, cudaStreamSynchronize(k->stream));
    int32_t c[2];
    KCUDA(k, cudaMemcpy(c, k->D.cnt + I_NE, sizeof c, cudaMemcpyDeviceToHost));
    if (c[0] > e_cap || c[1] > h_cap) return kfail(k, LGM_ERR_CAPACITY, "buffers too small");
    if (c[0]) KCUDA(k, cudaMemcpy(e, k->D.e_site, sizeof(int32_t) * c[0], cudaMemcpyDeviceToHost));
    if (c[1]) KCUDA(k, cudaMemcpy(h, k->D.h_site, sizeof(int32_t) * c[1], cudaMemcpyDeviceToHost));
    return LGM_OK;
}

lgm_status lgm_kmc_set_carriers(lgm_kmc* k, const int32_t* e, int32_t ne, const int32_t* h,
                                int32_t nh) {
    if (!k || ne < 0 || nh < 0 || (ne && !e) || (nh && !h)) return LGM_ERR_INVALID_ARGUMENT;
    if (ne > k->max_e || nh > k->max_h) return kfail(k, LGM_ERR_CAPACITY, "more carriers than the maxima");
    KCUDA(k, cudaSetDevice(k->device));
    KCUDA(k, cudaStreamSynchronize(k->stream));
    return upload_carriers(k, e, ne, h, nh);
}

lgm_status lgm_kmc_get_world(lgm_kmc* k, double* pot, int32_t* defects, int32_t d_cap,
                             int32_t* traps, double* trap_pots, int32_t t_cap) {
    if (!k) return LGM_ERR_INVALID_ARGUMENT;
    if (pot) std::memcpy(pot, k->pot.data(), sizeof(double) * k->V);
    if (defects) {
        if ((int)k->defects.size() > d_cap) return kfail(k, LGM_ERR_CAPACITY, "defect buffer too small");
        std::memcpy(defects, k->defects.data(), sizeof(int32_t) * k->defects.size());
    }
    if (traps || trap_pots) {
        if ((int)k->traps.size() > t_cap) return kfail(k, LGM_ERR_CAPACITY, "trap buffer too small");
        if (traps) std::memcpy(traps, k->traps.data(), sizeof(int32_t) * k->traps.size());
        if (trap_pots) std::memcpy(trap_pots, k->trap_pots.data(), sizeof(double) * k->traps.size());
    }
    return LGM_OK;
}

lgm_status lgm_kmc_set_morphology(lgm_kmc* k, const uint8_t* phase) {
    if (!k || !phase) return LGM_ERR_INVALID_ARGUMENT;
    KCUDA(k, cudaSetDevice(k->device));
    KCUDA(k, cudaStreamSynchronize(k->stream));
    const Dev& D = k->D;
    for (int s = 0; s < k->V; ++s)
        if (phase[s] > 1) return kfail(k, LGM_ERR_INVALID_ARGUMENT, "phase values must be 0 or 1");
    KCUDA(k, cudaMemcpy(D.phase, phase, k->V, cudaMemcpyHostToDevice));
    int32_t nb = 0;
    if (D.gen_iface) {
        // donor-acceptor bonds, from each donor site in site order over its
        // range-1 lattice neighbours in the order of Grid::neighborsSite
        std::vector<int32_t> bonds;
        const int X = D.X, Y = D.Y, Z = D.Z;
        for (int s = 0; s < k->V; ++s) {
            if (phase[s] != 0) continue;
            const int z = s / D.XY, y = s / X - z * Y, x = s % X;
            const int cand[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z},
                                    {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
            for (const auto& c : cand) {
                if (c[0] < 0 || c[0] >= X || c[1] < 0 || c[1] >= Y || c[2] < 0 || c[2] >= Z) continue;
                const int t = X * (c[1] + c[2] * Y) + c[0];
                if (phase[t] == 1) { bonds.push_back(s); bonds.push_back(t); }
            }
        }
        nb = (int32_t)(bonds.size() / 2);
        if (nb) KCUDA(k, cudaMemcpy(D.bonds, bonds.data(), sizeof(int32_t) * bonds.size(),
                                    cudaMemcpyHostToDevice));
    }
    KCUDA(k, cudaMemcpy(D.cnt + I_NBONDS, &nb, sizeof nb, cudaMemcpyHostToDevice));
    return LGM_OK;
}

lgm_status lgm_kmc_last_outcomes(lgm_kmc* k, int32_t* outcome, double* de, int32_t cap) {
    if (!k) return LGM_ERR_INVALID_ARGUMENT;
    KCUDA(k, cudaStreamSynchronize(k->stream));
    int32_t c[2];
    KCUDA(k, cudaMemcpy(c, k->D.cnt + I_NE0, sizeof c, cudaMemcpyDeviceToHost));
    const int n = c[0] + c[1];
    if (n > cap) return kfail(k, LGM_ERR_CAPACITY, "buffer too small");
    if (n && outcome) KCUDA(k, cudaMemcpy(outcome, k->D.outcome, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    if (n && de) KCUDA(k, cudaMemcpy(de, k->D.de, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return LGM_OK;
}

}  // extern "C"

// ---- batched replicas ----------------------------------------------------------------
//
// Many independent replicas of uneven size advance together: every phase of
// the step is one launch over all replicas (a block-to-replica map for the
// per-carrier phases, a work-item table of (replica, tile, split) for the
// pair sums), and the whole batched step is one CUDA graph.  Replica i keeps
// the Philox key of a single replica with id replica0 + i, so a batched run
// reproduces the single-replica runs bit for bit.

namespace {

struct BatchVariant {
    int nt, rp;
    void (*fn[2])(const PairArgs*, const int4*);
};
#define LGM_BV(NT, RP)                                                                 \
    BatchVariant {                                                                     \
        NT, RP, {                                                                      \
            &pair_kernel_items<0, 0, NT, RP, kSUB, true, true>,                        \
                &pair_kernel_items<1, 0, NT, RP, kSUB, true, true>                     \
        }                                                                              \
    }
const BatchVariant kBatchVariants[] = {LGM_BV(128, 4), LGM_BV(128, 2), LGM_BV(64, 4),
                                       LGM_BV(256, 2)};
constexpr int kNumBatchVariants = 4;
// Source chunks per pair work item tried by the tuner.
const int kChunksPerItem[] = {16, 48};
// A batch whose replicas all have room for at most this many charges takes
// the fused step by default (one block per replica).
constexpr int kFusedMaxCharges = 2048;
// Steps per launch of the fused kernel when no replica needs the per-phase
// kernels (bounds the length of one launch).
constexpr int kFusedStepsPerLaunch = 1000;

}  // namespace

struct lgm_kmc_batch {
    std::vector<lgm_kmc*> reps;
    int device = 0;
    int gauss = 0;
    int coulomb = 0;
    int recomb = 0;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    Dev* d_reps = nullptr;
    PairArgs* d_pargs = nullptr;
    int4* d_items = nullptr;
    int n_items = 0;
    int4 *map_car = nullptr, *map_pack = nullptr, *map_fin = nullptr, *map_guard = nullptr;
    int4* map_bins = nullptr;  // the target sort's bin counters
    int nb_car = 0, nb_pack = 0, nb_fin = 0, nb_guard = 0, nb_bins = 0;
    int compact_threads = kCompactThreads;  // block size of the per-replica list compaction
    // replicas on the fused step and on the per-phase kernels
    int fused_max = kFusedMaxCharges;
    bool started = false;  // a step has run: the partition is fixed
    bool fused_small = false;  // every fused replica fits the 128-thread block
    bool fused_set = false;    // the caller set the bound: capacity alone decides
    std::vector<int> fused, classic;
    int *d_fused = nullptr, *d_classic = nullptr;
    // per-phase replicas whose pair sum culls source chunks (point charges):
    // their chunk boxes, tile culls and one persistent launch over all their
    // work items (lgm_cull.cuh, ProblemList); the others take the items kernel
    std::vector<int> culled;
    int* d_culled = nullptr;
    int32_t* d_coffs = nullptr;      // [culled + 2] work-item offsets, next item taken
    int32_t* d_chist = nullptr;      // [kCostBuckets] the culled items' costs
    int32_t* d_corder = nullptr;     // the culled items, largest first
    PairArgs* d_cpargs = nullptr;    // [count], filled for the culled replicas
    CullArgs* d_cargs = nullptr;     // [count]
    int2 *map_box = nullptr, *map_cull = nullptr;
    int nb_box = 0, nb_cull = 0, cull_grid = 0;
    cudaStream_t aux = nullptr;            // the fused branch of the graph
    cudaEvent_t fork = nullptr, join = nullptr;
    DevicePool pool;                         // every replica's buffers
    int variant = 0, cpi = 16;
    std::vector<Dev> hD;
    std::string err;
};

namespace {

thread_local std::string g_batch_create_error;

lgm_status bfail(lgm_kmc_batch* b, lgm_status s, const std::string& m) {
    if (b) b->err = m;
    return s;
}

#define BCUDA(b, call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return bfail((b), LGM_ERR_CUDA, std::string(#call ": ") + \
                                                               cudaGetErrorString(e_));  \
    } while (0)

// Pair work items and per-replica split counts for a variant / chunk budget.
lgm_status build_items(lgm_kmc_batch* b, int v, int cpi) {
    const BatchVariant& BV = kBatchVariants[v];
    const int tile = BV.nt * 2 * BV.rp;
    std::vector<int4> items;
    std::vector<float> cost;  // source chunks an item streams (capacity estimate)
    std::vector<PairArgs> pargs(b->reps.size());
    for (int r : b->fused) b->hD[r].splits = 1;  // the fused pair sum is one split
    for (int r : b->classic) {
        Dev& D = b->hD[r];
        if (D.culled) continue;  // the culled launch covers it
        const lgm_kmc* k = b->reps[r];
        const int chunks = D.src_cap / CH;
        const int splits = std::max(1, std::min(k->D.splits, (chunks + cpi - 1) / cpi));
        D.splits = splits;
        const int tiles = (D.nterms * D.tpad_cap + tile - 1) / tile;
        for (int t = 0; t < tiles; ++t)
            for (int sp = 0; sp < splits; ++sp) items.push_back(make_int4(r, t, sp, splits));
        cost.resize(items.size(), (float)chunks / splits);
        PairArgs& A = pargs[r];
        A.geo = D.geo; A.qq = D.qq; A.splits = splits; A.tgt = D.tgt; A.part = D.part;
        A.part_norm = D.part_norm; A.c2 = (float)D.cutoff2;
        A.tab = k->gtab; A.tab_k = D.gauss ? k->gtab_k : 0;
        A.err = D.err; A.dyn = D.cnt + I_NCHUNK;
    }
    // Longest items first: the block scheduler hands out blocks in index
    // order, so the long items of the large replicas start in the first wave
    // and the short ones fill in behind them.  The order does not change any
    // sum (each item writes its own partials).
    {
        std::vector<int> ord(items.size());
        for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return cost[x] > cost[y]; });
        std::vector<int4> sorted(items.size());
        for (size_t i = 0; i < ord.size(); ++i) sorted[i] = items[ord[i]];
        items.swap(sorted);
    }
    if (b->d_items) cudaFree(b->d_items);
    b->d_items = nullptr;
    BCUDA(b, cudaMalloc(&b->d_items, sizeof(int4) * std::max<size_t>(items.size(), 1)));
    if (!items.empty())
        BCUDA(b, cudaMemcpy(b->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
    BCUDA(b, cudaMemcpy(b->d_pargs, pargs.data(), sizeof(PairArgs) * pargs.size(), cudaMemcpyHostToDevice));
    BCUDA(b, cudaMemcpy(b->d_reps, b->hD.data(), sizeof(Dev) * b->hD.size(), cudaMemcpyHostToDevice));
    b->n_items = (int)items.size();
    return LGM_OK;
}

size_t batch_smem(const lgm_kmc_batch* b) {
    int tk = 0;
    for (const lgm_kmc* k : b->reps) tk = std::max(tk, k->D.gauss ? k->gtab_k : 0);
    return pair_smem_bytes(tk);
}

// The work-item kernel over the per-phase replicas that do not cull.
lgm_status enqueue_batch_items(lgm_kmc_batch* b, cudaStream_t st) {
    if (b->n_items > 0) {
        const BatchVariant& BV = kBatchVariants[b->variant];
        BV.fn[b->gauss]<<<b->n_items, BV.nt, batch_smem(b), st>>>(b->d_pargs, b->d_items);
    }
    BCUDA(b, cudaGetLastError());
    return LGM_OK;
}

// The batched pair sum: the culled replicas' chunk boxes, tile culls, item
// offsets and one persistent launch over all their items, then the work-item
// kernel over the rest.
lgm_status enqueue_batch_pair(lgm_kmc_batch* b, cudaStream_t st) {
    if (!b->culled.empty()) {
        const int n = (int)b->culled.size();
        kb_chunk_boxes<<<b->nb_box, CH, 0, st>>>(b->d_reps, b->map_box);
        kb_cull<<<b->nb_cull, kCullThreads, 0, st>>>(b->d_reps, b->map_cull);
        kb_item_order<<<1, 1024, 0, st>>>(
            ProblemList{b->d_cpargs, b->d_cargs, b->d_culled, b->d_coffs, n, nullptr}, b->d_reps,
            b->d_chist, b->d_coffs, b->d_corder);
        kBatchCulled<<<b->cull_grid, kCThreads, kmc_culled_smem(0), st>>>(
            ProblemList{b->d_cpargs, b->d_cargs, b->d_culled, b->d_coffs, n, b->d_corder});
    }
    return enqueue_batch_items(b, st);
}

void launch_fused(const lgm_kmc_batch* b, cudaStream_t st, int steps) {
    const int n = (int)b->fused.size();
    if (b->fused_small)
        kb_fused<128><<<n, 128, 0, st>>>(b->d_reps, b->d_fused, steps, b->recomb);
    else
        kb_fused<256><<<n, 256, 0, st>>>(b->d_reps, b->d_fused, steps, b->recomb);
}

// The fused replicas' step on the aux stream, forked from and joined back to
// the batch stream (inside a capture: a parallel branch of the graph).
lgm_status enqueue_fused(lgm_kmc_batch* b, int steps, bool branch) {
    if (b->fused.empty()) return LGM_OK;
    cudaStream_t st = b->stream;
    if (branch) {
        BCUDA(b, cudaEventRecord(b->fork, b->stream));
        BCUDA(b, cudaStreamWaitEvent(b->aux, b->fork, 0));
        st = b->aux;
    }
    launch_fused(b, st, steps);
    BCUDA(b, cudaGetLastError());
    if (branch) {
        BCUDA(b, cudaEventRecord(b->join, b->aux));
        BCUDA(b, cudaStreamWaitEvent(b->stream, b->join, 0));
    }
    return LGM_OK;
}

// The per-phase replicas' targets in lattice-cell order (before pack).
void enqueue_batch_sort(lgm_kmc_batch* b, cudaStream_t st) {
    kb_tbins_zero<<<b->nb_bins, 256, 0, st>>>(b->d_reps, b->map_bins);
    kb_tbins<<<b->nb_fin, 256, 0, st>>>(b->d_reps, b->map_fin);
    kb_tbins_scan<<<dim3((unsigned)b->classic.size(), b->culled.empty() ? 1u : 2u), 1024, 0, st>>>(
        b->d_reps, b->d_classic);
    kb_tscatter<<<b->nb_fin, 256, 0, st>>>(b->d_reps, b->map_fin);
    if (!b->culled.empty()) kb_trank<<<b->nb_fin, 256, 0, st>>>(b->d_reps, b->map_fin);
}

lgm_status enqueue_batch_step(lgm_kmc_batch* b) {
    cudaStream_t st = b->stream;
    if (b->classic.empty()) return enqueue_fused(b, 1, false);
    const bool fork = !b->fused.empty();
    if (fork) {
        BCUDA(b, cudaEventRecord(b->fork, b->stream));
        BCUDA(b, cudaStreamWaitEvent(b->aux, b->fork, 0));
        launch_fused(b, b->aux, 1);
        BCUDA(b, cudaGetLastError());
    }
    const int R = (int)b->classic.size();
    kb_choose<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    if (b->coulomb) {
        enqueue_batch_sort(b, st);
        kb_pack<<<b->nb_pack, 256, 0, st>>>(b->d_reps, b->map_pack);
        lgm_status s = enqueue_batch_pair(b, st);
        if (s != LGM_OK) return s;
        kb_finalize<<<b->nb_fin, 256, 0, st>>>(b->d_reps, b->map_fin);
    }
    kb_decide<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    if (b->coulomb) kb_guard<<<b->nb_guard, kGuardThreadsBatch, 0, st>>>(b->d_reps, b->map_guard);
    if (b->recomb) {
        kb_hmap<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
        kb_recomb_propose<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
        kb_recomb_resolve<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
        kb_recomb_reset<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    }
    kb_claim<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    kb_move<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    kb_unclaim<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    kb_compact_inject<<<R, b->compact_threads, 0, st>>>(b->d_reps, b->d_classic);
    BCUDA(b, cudaGetLastError());
    if (fork) {
        BCUDA(b, cudaEventRecord(b->join, b->aux));
        BCUDA(b, cudaStreamWaitEvent(b->stream, b->join, 0));
    }
    return LGM_OK;
}

// The project's tile tuner for the batch: times every (variant, chunks per
// item) pair on the batch's current charges with CUDA events, keeps the best.
lgm_status tune_batch(lgm_kmc_batch* b) {
    if (!b->coulomb || b->classic.size() == b->culled.size()) return LGM_OK;
    cudaStream_t st = b->stream;
    kb_choose<<<b->nb_car, 256, 0, st>>>(b->d_reps, b->map_car);
    enqueue_batch_sort(b, st);
    kb_pack<<<b->nb_pack, 256, 0, st>>>(b->d_reps, b->map_pack);
    BCUDA(b, cudaGetLastError());
    cudaEvent_t e0, e1;
    BCUDA(b, cudaEventCreate(&e0));
    BCUDA(b, cudaEventCreate(&e1));
    float best = 1e30f;
    int bv = 0, bc = kChunksPerItem[0];
    for (int v = 0; v < kNumBatchVariants; ++v)
        for (int cpi : kChunksPerItem) {
            b->variant = v;
            lgm_status s = build_items(b, v, cpi);
            if (s != LGM_OK) return s;
            float ms[3];
            for (int r = 0; r < 3; ++r) {
                cudaEventRecord(e0, st);
                if ((s = enqueue_batch_items(b, st)) != LGM_OK) return s;
                cudaEventRecord(e1, st);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms[r], e0, e1);
            }
            std::sort(ms, ms + 3);
            if (ms[1] < best) { best = ms[1]; bv = v; bc = cpi; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->variant = bv;
    b->cpi = bc;
    // the step counters advanced by nothing: choose/pack only snapshot counts
    return build_items(b, bv, bc);
}

// Splits the replicas between the fused step (room for at most b->fused_max
// charges) and the per-phase kernels, and builds the per-phase kernels' block
// maps -- {replica, local block, blocks of the replica, index bound} -- and
// pair work items over the latter.
lgm_status partition_batch(lgm_kmc_batch* b) {
    b->fused.clear();
    b->classic.clear();
    // By default a batch takes one form: the fused step when every replica fits
    // one block, else the per-phase kernels for all (beside a graph of large
    // replicas the fused blocks measured slower than the per-phase kernels on
    // the same small replicas).  A bound set by the caller splits the batch.
    bool all_fit = true;
    for (const Dev& D : b->hD) all_fit &= D.cap_e + D.cap_h <= b->fused_max;
    for (int r = 0; r < (int)b->hD.size(); ++r) {
        const Dev& D = b->hD[r];
        const bool fits = D.cap_e + D.cap_h <= b->fused_max && (b->fused_set || all_fit);
        (fits ? b->fused : b->classic).push_back(r);
    }
    b->fused_small = true;
    for (int r : b->fused)
        b->fused_small &= b->hD[r].cap_e + b->hD[r].cap_h <= kFusedSmallCharges;
    for (int r : b->fused) b->hD[r].sorted = 0;  // the fused step keeps the list order
    for (int r : b->classic) b->hD[r].sorted = b->hD[r].coulomb;
    // culled pair sums for the per-phase replicas with room for enough chunks
    // (point charges: the Gaussian tables differ between replicas)
    b->culled.clear();
    for (int r = 0; r < (int)b->hD.size(); ++r) {
        b->hD[r].culled = 0;
        b->hD[r].chist = b->reps[r]->D.chist;
        b->hD[r].corder = b->reps[r]->D.corder;
    }
    for (int r : b->classic)
        if (b->reps[r]->cull_ok && !b->gauss) {
            b->hD[r].culled = 1;
            b->culled.push_back(r);
        }
    // the culled items' cost histogram and order are the batch's
    for (int32_t** p : {&b->d_coffs, &b->d_chist, &b->d_corder}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    size_t order_cap = 1;
    for (int r : b->culled) order_cap += (size_t)b->reps[r]->cull_tiles * b->hD[r].max_items;
    if (cudaMalloc(&b->d_coffs, sizeof(int32_t) * (b->culled.size() + 2)) != cudaSuccess ||
        cudaMalloc(&b->d_chist, sizeof(int32_t) * kCostBuckets) != cudaSuccess ||
        cudaMalloc(&b->d_corder, sizeof(int32_t) * order_cap) != cudaSuccess)
        return bfail(b, LGM_ERR_CUDA, "work-item offsets");
    std::vector<int2> box, cull;
    std::vector<PairArgs> cpargs(b->hD.size());
    std::vector<CullArgs> cargs(b->hD.size());
    for (int r : b->culled) {
        Dev& D = b->hD[r];
        D.chist = b->d_chist;
        D.corder = nullptr;
        for (int c = 0; c < D.src_cap / CH; ++c) box.push_back(make_int2(r, c));
        for (int t = 0; t < b->reps[r]->cull_tiles; ++t) cull.push_back(make_int2(r, t));
        cpargs[r] = pair_args(D);
        cargs[r] = cull_args(D);
    }
    std::vector<int4> car, pack, fin, guard, bins;
    auto add = [](std::vector<int4>& v, int r, int bound) {
        const int nb = std::max(1, (bound + kItemsPerThread * 256 - 1) / (kItemsPerThread * 256));
        for (int i = 0; i < nb; ++i) v.push_back(make_int4(r, i, nb, bound));
    };
    int max_cap = 1;
    for (int r : b->classic) {
        const Dev& D = b->hD[r];
        const int ncap = std::max(1, D.cap_e + D.cap_h);
        add(car, r, ncap);
        add(pack, r, std::max(D.src_cap, D.tpad_cap));
        // a culled replica's source sort also walks the defects
        add(fin, r, D.culled ? std::max(2 * ncap, ncap + (D.dq != 0 ? D.nd : 0)) : 2 * ncap);
        add(bins, r, D.culled ? 3 * (D.ncells + 1) : D.ncells + 1);
        // flagged decisions grow with the charge count: one block per 512 of capacity
        const int ng = std::min(kGuardBlocksPerReplica, std::max(1, (ncap + 511) / 512));
        for (int i = 0; i < ng; ++i) guard.push_back(make_int4(r, i, ng, 0));
        max_cap = std::max(max_cap, std::max(D.cap_e, D.cap_h));
    }
    auto upload = [&](auto** dst, const auto& v) -> bool {
        if (*dst) cudaFree(*dst);
        *dst = nullptr;
        const size_t bytes = sizeof(v[0]) * std::max<size_t>(v.size(), 1);
        return cudaMalloc(dst, bytes) == cudaSuccess &&
               (v.empty() || cudaMemcpy(*dst, v.data(), sizeof(v[0]) * v.size(),
                                        cudaMemcpyHostToDevice) == cudaSuccess);
    };
    if (!upload(&b->map_car, car) || !upload(&b->map_pack, pack) || !upload(&b->map_fin, fin) ||
        !upload(&b->map_guard, guard) || !upload(&b->map_bins, bins) ||
        !upload(&b->d_fused, b->fused) || !upload(&b->d_classic, b->classic) ||
        !upload(&b->d_culled, b->culled) || !upload(&b->map_box, box) ||
        !upload(&b->map_cull, cull) || !upload(&b->d_cpargs, cpargs) ||
        !upload(&b->d_cargs, cargs))
        return bfail(b, LGM_ERR_CUDA, "block maps");

    b->nb_box = (int)box.size();
    b->nb_cull = (int)cull.size();
    if (!b->culled.empty()) {
        int dev_sms = 0, cbps = 1;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, b->device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cbps, kBatchCulled, kCThreads,
                                                      kmc_culled_smem(0));
        b->cull_grid = std::max(1, dev_sms) * std::max(1, cbps);
    }
    b->nb_guard = (int)guard.size();
    b->nb_bins = (int)bins.size();
    // the compaction loops over its list in blocks: small replicas need no 1024-thread block
    b->compact_threads = max_cap > 4096 ? kCompactThreads : 256;
    b->nb_car = (int)car.size();
    b->nb_pack = (int)pack.size();
    b->nb_fin = (int)fin.size();
    return build_items(b, 0, kChunksPerItem[0]);
}

}  // namespace

extern "C" {

lgm_status lgm_kmc_batch_create(const lgm_params* params, int32_t count, int32_t device,
                                uint32_t replica0, lgm_kmc_batch** out) {
    g_batch_create_error.clear();
    if (!params || count < 1 || !out) return LGM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    lgm_kmc_batch* b = new (std::nothrow) lgm_kmc_batch();
    if (!b) return LGM_ERR_INVALID_ARGUMENT;
    auto bail = [&](lgm_status s, const std::string& m) {
        g_batch_create_error = m;
        lgm_kmc_batch_destroy(b);
        return s;
    };
    b->device = device < 0 ? 0 : device;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(LGM_ERR_CUDA, "stream");
    // replicas share the batch's stream and take their buffers from its pool
    for (int i = 0; i < count; ++i) {
        lgm_kmc* k = nullptr;
        lgm_status s = kmc_create_impl(&params[i], b->device, replica0 + (uint32_t)i, &k,
                                       &b->pool, b->stream);
        if (s != LGM_OK) return bail(s, "replica " + std::to_string(i) + ": " + lgm_kmc_last_error(nullptr));
        b->reps.push_back(k);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(LGM_ERR_CUDA, "replica set-up");
    // one interaction kind and one cutoff-table layout per batch
    b->gauss = b->reps[0]->D.gauss;
    b->coulomb = b->reps[0]->D.coulomb;
    for (lgm_kmc* k : b->reps) b->recomb |= (k->D.solar && k->D.rec_rate > 0);
    for (lgm_kmc* k : b->reps)
        if (k->D.gauss != b->gauss || k->D.coulomb != b->coulomb)
            return bail(LGM_ERR_UNSUPPORTED,
                        "a batch mixes point and Gaussian charges or Coulomb on and off");
    for (lgm_kmc* k : b->reps) b->hD.push_back(k->D);
    if (cudaMalloc(&b->d_reps, sizeof(Dev) * count) != cudaSuccess ||
        cudaMalloc(&b->d_pargs, sizeof(PairArgs) * count) != cudaSuccess)
        return bail(LGM_ERR_CUDA, "descriptors");
    if (b->gauss) {
        cudaFuncSetAttribute(kBatchVariants[0].fn[1], cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)batch_smem(b));
        for (const BatchVariant& BV : kBatchVariants)
            cudaFuncSetAttribute(BV.fn[1], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)batch_smem(b));
    }
    if (cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming) != cudaSuccess)
        return bail(LGM_ERR_CUDA, "fused branch stream");
    lgm_status s = partition_batch(b);
    if (s != LGM_OK) return bail(s, b->err);
    *out = b;
    return LGM_OK;
}

lgm_status lgm_kmc_batch_destroy(lgm_kmc_batch* b) {
    if (!b) return LGM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    void* ptrs[] = {b->d_reps, b->d_pargs, b->d_items, b->map_car, b->map_pack, b->map_fin,
                    b->map_guard, b->map_bins, b->d_fused, b->d_classic, b->d_culled,
                    b->d_coffs, b->d_cpargs, b->d_cargs, b->map_box, b->map_cull,
                    b->d_chist, b->d_corder};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->aux) cudaStreamDestroy(b->aux);
    for (lgm_kmc* k : b->reps) lgm_kmc_destroy(k);  // they do not own the stream or pool
    if (b->stream) cudaStreamDestroy(b->stream);
    b->pool.release();
    delete b;
    return LGM_OK;
}

const char* lgm_kmc_batch_last_error(const lgm_kmc_batch* b) {
    return b ? b->err.c_str() : g_batch_create_error.c_str();
}

int32_t lgm_kmc_batch_size(const lgm_kmc_batch* b) { return b ? (int32_t)b->reps.size() : 0; }

int32_t lgm_kmc_batch_culled_count(const lgm_kmc_batch* b) {
    return b ? (int32_t)b->culled.size() : 0;
}

lgm_kmc* lgm_kmc_batch_replica(lgm_kmc_batch* b, int32_t i) {
    if (!b || i < 0 || i >= (int)b->reps.size()) return nullptr;
    return b->reps[i];
}

lgm_status lgm_kmc_batch_run(lgm_kmc_batch* b, int32_t steps) {
    if (!b || steps < 0) return LGM_ERR_INVALID_ARGUMENT;
    BCUDA(b, cudaSetDevice(b->device));
    BCUDA(b, cudaStreamSynchronize(b->stream));  // every replica's work is on the batch stream
    b->started = true;
    if (b->classic.empty()) {
        // every replica on the fused step: many steps per launch, no graph needed
        for (int done = 0; done < steps; done += kFusedStepsPerLaunch) {
            lgm_status s = enqueue_fused(b, std::min(kFusedStepsPerLaunch, steps - done), false);
            if (s != LGM_OK) return s;
        }
        BCUDA(b, cudaStreamSynchronize(b->stream));
        return LGM_OK;
    }
    if (!b->exec && steps > 0) {
        lgm_status s = tune_batch(b);
        if (s != LGM_OK) return s;
        BCUDA(b, cudaStreamSynchronize(b->stream));
        BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        s = enqueue_batch_step(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (s != LGM_OK) { if (g) cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) return bfail(b, LGM_ERR_CUDA, "graph capture failed");
        b->graph = g;
        BCUDA(b, cudaGraphInstantiate(&b->exec, g, 0));
    }
    for (int i = 0; i < steps; ++i) BCUDA(b, cudaGraphLaunch(b->exec, b->stream));
    BCUDA(b, cudaStreamSynchronize(b->stream));
    return LGM_OK;
}

lgm_status lgm_kmc_batch_set_fused(lgm_kmc_batch* b, int32_t max_charges) {
    if (!b || max_charges < 0) return LGM_ERR_INVALID_ARGUMENT;
    if (b->started) return bfail(b, LGM_ERR_INVALID_ARGUMENT, "set before the first step");
    BCUDA(b, cudaSetDevice(b->device));
    b->fused_max = max_charges;
    b->fused_set = true;
    return partition_batch(b);
}

int32_t lgm_kmc_batch_fused_count(const lgm_kmc_batch* b) {
    return b ? (int32_t)b->fused.size() : 0;
}

lgm_status lgm_kmc_batch_time_pair(lgm_kmc_batch* b, int32_t reps, float* ms) {
    if (!b || reps < 1 || !ms) return LGM_ERR_INVALID_ARGUMENT;
    if (!b->exec || !b->coulomb || b->classic.empty())
        return bfail(b, LGM_ERR_STATE, "no per-phase Coulomb step has run");
    BCUDA(b, cudaSetDevice(b->device));
    cudaStream_t st = b->stream;
    BCUDA(b, cudaStreamSynchronize(st));
    cudaEvent_t e0, e1;
    BCUDA(b, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return bfail(b, LGM_ERR_CUDA, "cudaEventCreate");
    }
    std::vector<float> t(reps);
    lgm_status s = LGM_OK;
    for (int r = 0; r < reps && s == LGM_OK; ++r) {
        cudaEventRecord(e0, st);
        s = enqueue_batch_pair(b, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) s = bfail(b, LGM_ERR_CUDA, "pair launch");
        cudaEventElapsedTime(&t[r], e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != LGM_OK) return s;
    std::sort(t.begin(), t.end());
    *ms = t[reps / 2];
    return LGM_OK;
}

lgm_status lgm_kmc_batch_count_pairs(lgm_kmc_batch* b, uint64_t* pairs) {
    if (!b || !pairs) return LGM_ERR_INVALID_ARGUMENT;
    if (!b->exec || !b->coulomb || b->classic.empty())
        return bfail(b, LGM_ERR_STATE, "no per-phase Coulomb step has run");
    BCUDA(b, cudaSetDevice(b->device));
    cudaStream_t st = b->stream;
    BCUDA(b, cudaStreamSynchronize(st));
    unsigned long long* d_n = nullptr;
    BCUDA(b, cudaMalloc(&d_n, sizeof *d_n));
    std::vector<CullArgs> cargs(b->hD.size());
    for (int r : b->culled) {
        cargs[r] = cull_args(b->hD[r]);
        cargs[r].examined = d_n;
    }
    lgm_status s = LGM_OK;
    unsigned long long h = 0;
    auto put = [&](bool on) {
        if (!on)
            for (int r : b->culled) cargs[r].examined = nullptr;
        return cudaMemcpy(b->d_cargs, cargs.data(), sizeof(CullArgs) * cargs.size(),
                          cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (cudaMemset(d_n, 0, sizeof *d_n) != cudaSuccess || !put(true)) {
        s = bfail(b, LGM_ERR_CUDA, "pair counter");
    } else {
        s = enqueue_batch_pair(b, st);
        if (s == LGM_OK) {
            kb_tested_pairs<<<1, 256, 0, st>>>(b->d_reps, b->d_classic, (int)b->classic.size(), d_n);
            if (cudaStreamSynchronize(st) != cudaSuccess ||
                cudaMemcpy(&h, d_n, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess)
                s = bfail(b, LGM_ERR_CUDA, "pair count");
        }
        if (!put(false) && s == LGM_OK) s = bfail(b, LGM_ERR_CUDA, "pair counter");
    }
    cudaFree(d_n);
    if (s == LGM_OK) *pairs = h;
    return s;
}

lgm_status lgm_kmc_batch_tuning(const lgm_kmc_batch* b, int32_t* threads, int32_t* target_pairs,
                                int32_t* chunks_per_item, int32_t* items) {
    if (!b) return LGM_ERR_INVALID_ARGUMENT;
    if (threads) *threads = kBatchVariants[b->variant].nt;
    if (target_pairs) *target_pairs = kBatchVariants[b->variant].rp;
    if (chunks_per_item) *chunks_per_item = b->cpi;
    if (items) *items = b->n_items;
    return LGM_OK;
}

}  // extern "C"
