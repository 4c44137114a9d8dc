// lgm_oracle_kmc.cpp -- CPU FP64 oracle of one kMC step (TEST INFRASTRUCTURE).
//
// Restates Simulation::performIterations for the transistor set-up
// (simulation.cpp:34-111): chooseFuture for every electron then hole
// (chargeagent.cpp:73-78), the Coulomb energy change of ChargeAgent::coulombCPU
// (chargeagent.cpp:215-271), decideFuture (chargeagent.cpp:90-161) with
// Random::metropolisWithCoupling (rand.cpp:91-106) and DrainAgent::tryToAccept
// (drainagent.cpp:83-92), nextTick / completeTick in list order
// (simulation.cpp:355-414, chargeagent.cpp:163-199) and the four electrode
// sources' tryToInject (sourceagent.cpp:92-103, 204-232).
//
// Random numbers: the reference draws from one serial Boost mt19937 stream;
// here every draw comes from Philox4x32-10 at a counter named by (step,
// list index, purpose) -- the stream the GPU step uses too, so decisions can
// be compared bit for bit.  Layout (shared with langmuir_b200/csrc/lgm_rng.cuh):
//   key = {seed, replica},  counter = {step, index, purpose, 0}
//   purpose 1/2: choose/decide of electron `index`, 3/4: of hole `index`,
//   5: recombination of electron `index` (w0: candidate, (w1, w2): accept),
//   16 + k: electrode source k (0 eL, 1 eR, 2 hL, 3 hR), 20: exciton source,
//   index 0.
//   integer in [0, n): (w0 * n) >> 32;  uniform [0,1): ((w_a >> 5) 2^26 + (w_b >> 6)) / 2^53
//   with (a, b) = (0, 1) for decisions and (1, 2) for sources.
#include <cmath>
#include <cstring>
#include <vector>

#include "lgm_oracle.h"

namespace {

struct Draw {
    uint32_t w[4];
};

Draw draw(const orc_kmc_config* k, uint32_t step, uint32_t index, uint32_t purpose) {
    const uint32_t ctr[4] = {step, index, purpose, 0u};
    const uint32_t key[2] = {k->seed, k->replica};
    Draw d;
    orc_philox4x32_10(ctr, key, d.w);
    return d;
}

inline uint32_t uint_below(uint32_t w, uint32_t n) {
    return (uint32_t)(((uint64_t)w * n) >> 32);
}

inline double unit_double(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// Special-agent ids (Grid::registerSpecialAgent, cubicgrid.cpp:558-589, in
// the creation order of World::createSources/createDrains, world.cpp:961-1187):
// electron grid V+0 eSourceL, V+1 eSourceR, V+2 exciton source, V+3 eDrainL,
// V+4 eDrainR, V+5 recombination; hole grid V+0 hSourceL, V+1 hSourceR,
// V+2 hDrainL, V+3 hDrainR.
enum { E_DRAIN_L = 3, E_DRAIN_R = 4, H_DRAIN_L = 2, H_DRAIN_R = 3 };

}  // namespace

extern "C" int orc_kmc_step(const orc_ctx* ctx, const orc_kmc_config* k, const double* pot,
                            const int32_t* defects, int nd, uint32_t step, int32_t* e_site,
                            int32_t* ne_io, int32_t* h_site, int32_t* nh_io, uint64_t* counters,
                            int32_t* outcome, double* de_out, int threads) {
    int dims[3];
    orc_dims(ctx, dims);
    const int GX = dims[0], GY = dims[1], GZ = dims[2];
    const int V = GX * GY * GZ;
    const int hr = orc_hopping_range(ctx);
    int ne = *ne_io, nh = *nh_io;

    // Per-site agent types of both grids at the start of the step.
    std::vector<uint8_t> et(V + 35, ORC_EMPTY), ht(V + 35, ORC_EMPTY);
    for (int i = 0; i < nd; ++i) et[defects[i]] = ht[defects[i]] = ORC_DEFECT;
    for (int i = 0; i < ne; ++i) et[e_site[i]] = ORC_ELECTRON;
    for (int i = 0; i < nh; ++i) ht[h_site[i]] = ORC_HOLE;
    et[V + 0] = et[V + 1] = et[V + 2] = ORC_SOURCE;
    et[V + 3] = et[V + 4] = et[V + 5] = ORC_DRAIN;
    ht[V + 0] = ht[V + 1] = ORC_SOURCE;
    ht[V + 2] = ht[V + 3] = ORC_DRAIN;

    // chooseFuture (chargeagent.cpp:73-78) over Grid::neighborsSite
    // (cubicgrid.cpp:207-471): lattice neighbours, then the face drain.
    std::vector<int32_t> ef(ne), hf(nh);
    int nb[40];
    auto choose = [&](int site, bool electron, uint32_t index) {
        int n = orc_neighbors(ctx, site, hr, nb);
        const int x = orc_index_x(ctx, site);
        if (x == 0) nb[n++] = V + (electron ? E_DRAIN_L : H_DRAIN_L);
        if (x == GX - 1) nb[n++] = V + (electron ? E_DRAIN_R : H_DRAIN_R);
        const Draw d = draw(k, step, index, electron ? 1u : 3u);
        return nb[uint_below(d.w[0], (uint32_t)n)];
    };
    for (int i = 0; i < ne; ++i) ef[i] = choose(e_site[i], true, (uint32_t)i);
    for (int i = 0; i < nh; ++i) hf[i] = choose(h_site[i], false, (uint32_t)i);

    // Coulomb energy change (chargeagent.cpp:215-271), with the image sums as
    // an extension when requested.
    std::vector<double> de(ne + nh, 0.0);
    if (k->coulomb_carriers) {
        orc_coulomb_cpu(ctx, e_site, ef.data(), ne, h_site, hf.data(), nh, defects, nd,
                        k->defects_charge, et.data(), ht.data(), k->exciton_binding, de.data(),
                        nullptr, nullptr, threads);
        if (k->image_terms & 6u) {
            // p += image sums at both sites; de = q (dp2 - dp1)
            std::vector<int32_t> src, q;
            for (int i = 0; i < ne; ++i) { src.push_back(e_site[i]); q.push_back(-1); }
            for (int i = 0; i < nh; ++i) { src.push_back(h_site[i]); q.push_back(+1); }
            if (k->defects_charge != 0)
                for (int i = 0; i < nd; ++i) { src.push_back(defects[i]); q.push_back(k->defects_charge); }
            std::vector<int32_t> cur(ne + nh), fut(ne + nh);
            for (int i = 0; i < ne; ++i) { cur[i] = e_site[i]; fut[i] = ef[i]; }
            for (int i = 0; i < nh; ++i) { cur[ne + i] = h_site[i]; fut[ne + i] = hf[i]; }
            const unsigned it = k->image_terms & 6u;
            std::vector<double> i1(ne + nh), i2(ne + nh);
            orc_potentials(ctx, orc_sigma(ctx) > 0, it, src.data(), q.data(), (int)src.size(),
                           cur.data(), ne + nh, i1.data(), threads);
            orc_potentials(ctx, orc_sigma(ctx) > 0, it, src.data(), q.data(), (int)src.size(),
                           fut.data(), ne + nh, i2.data(), threads);
            for (int i = 0; i < ne + nh; ++i) de[i] += (i < ne ? -1.0 : 1.0) * (i2[i] - i1[i]);
        }
    }
    if (de_out) std::memcpy(de_out, de.data(), sizeof(double) * (ne + nh));

    // decideFuture (chargeagent.cpp:90-161).
    const double beta = k->inverse_kt;
    std::vector<double> coupling((hr + 1) * (hr + 1) * (hr + 1));
    orc_coupling_table(ctx, coupling.data());
    auto decide = [&](int site, int32_t& fsite, bool electron, uint32_t index, int32_t* code) {
        const std::vector<uint8_t>& own = electron ? et : ht;
        const int q = electron ? -1 : 1;
        uint8_t type = own[fsite];
        // extension: a carrier may not enter the other phase (treated as occupied)
        if (k->confine && k->phase && fsite < V && type == ORC_EMPTY &&
            k->phase[fsite] != (electron ? 1 : 0))
            type = ORC_DEFECT;
        if (type == ORC_EMPTY) {
            double pd = pot[fsite] - pot[site];
            pd *= q;
            pd += de[electron ? index : ne + index];
            const int dx = std::abs(orc_index_x(ctx, site) - orc_index_x(ctx, fsite));
            const int dy = std::abs(orc_index_y(ctx, site) - orc_index_y(ctx, fsite));
            const int dz = std::abs(orc_index_z(ctx, site) - orc_index_z(ctx, fsite));
            const double c = coupling[(dx * (hr + 1) + dy) * (hr + 1) + dz];
            const Draw d = draw(k, step, index, electron ? 2u : 4u);
            const double u = unit_double(d.w[0], d.w[1]);
            bool acc;
            if (pd > 0.0) acc = c * std::exp(-pd * beta) > u;  // rand.cpp:91-106
            else acc = c > u;
            if (!acc) fsite = site;
            *code = acc ? ORC_MET_ACCEPT : ORC_MET_REJECT;
        } else if (type == ORC_DRAIN) {
            const int which = fsite - V;  // drain id on this grid
            int agent;                    // counter slot 4..7: eDrainL, eDrainR, hDrainL, hDrainR
            double rate;
            if (electron) {
                agent = which == E_DRAIN_L ? 4 : 5;
                rate = which == E_DRAIN_L ? k->rate_e_drain_l : k->rate_e_drain_r;
            } else {
                agent = which == H_DRAIN_L ? 6 : 7;
                rate = which == H_DRAIN_L ? k->rate_h_drain_l : k->rate_h_drain_r;
            }
            counters[2 * agent] += 1;  // attempts
            const Draw d = draw(k, step, index, electron ? 2u : 4u);
            const double u = unit_double(d.w[0], d.w[1]);
            if (rate > u) {  // FluxAgent::shouldTransport -> chooseYes (fluxagent.cpp:125-130)
                counters[2 * agent + 1] += 1;
                *code = ORC_DRAIN_ACCEPT;
            } else {
                fsite = site;
                *code = ORC_DRAIN_REJECT;
            }
        } else {
            fsite = site;  // defect, same-type carrier (chargeagent.cpp:152-157)
            *code = ORC_OCCUPIED;
        }
    };
    std::vector<int32_t> codes(ne + nh, ORC_OCCUPIED);
    for (int i = 0; i < ne; ++i) decide(e_site[i], ef[i], true, (uint32_t)i, &codes[i]);
    for (int i = 0; i < nh; ++i) decide(h_site[i], hf[i], false, (uint32_t)i, &codes[ne + i]);
    if (outcome) std::memcpy(outcome, codes.data(), sizeof(int32_t) * (ne + nh));

    // performRecombinations (simulation.cpp:219-231), RecombinationAgent::tryToAccept
    // (drainagent.cpp:113-214) for every electron in list order.
    std::vector<uint8_t> e_rm(ne, 0), h_rm(nh, 0);
    if (k->solar && k->recombination_rate > 0) {
        std::vector<int32_t> h_at(V + 35, -1);
        for (int i = 0; i < nh; ++i) h_at[h_site[i]] = i;
        int rb[48];
        for (int i = 0; i < ne; ++i) {
            const int site = e_site[i];
            int n = 0;
            if (ht[site] == ORC_HOLE) rb[n++] = site;
            if (k->recombination_range > 0) {
                int nb2[40];
                int m = orc_neighbors(ctx, site, k->recombination_range, nb2);
                const int x = orc_index_x(ctx, site);
                // the electron's neighbour list carries its face drains too
                if (x == 0) nb2[m++] = V + E_DRAIN_L;
                if (x == GX - 1) nb2[m++] = V + E_DRAIN_R;
                for (int j = 0; j < m; ++j)
                    if (ht[nb2[j]] == ORC_HOLE) rb[n++] = nb2[j];
            }
            if (n == 0) continue;
            const Draw d = draw(k, step, (uint32_t)i, 5u);
            const int hs = rb[uint_below(d.w[0], (uint32_t)n)];
            const int hk = h_at[hs];
            if (h_rm[hk]) continue;  // already recombined
            counters[18] += 1;
            if (k->recombination_rate > unit_double(d.w[1], d.w[2])) {
                counters[19] += 1;
                e_rm[i] = 1;
                h_rm[hk] = 1;
            }
        }
    }

    // nextTick: completeTick in list order, first mover wins, drains remove.
    auto tick = [&](int32_t* site, const int32_t* fs, int n, std::vector<uint8_t>& own,
                    uint8_t mine, const std::vector<uint8_t>& rm) {
        int w = 0;
        for (int i = 0; i < n; ++i) {
            int s = site[i];
            bool removed = false;
            if (rm[i]) {  // completeTick: removed charges only leave (chargeagent.cpp:166-170)
                own[s] = ORC_EMPTY;
                continue;
            }
            if (s != fs[i]) {
                if (own[fs[i]] == ORC_EMPTY) {
                    own[s] = ORC_EMPTY;
                    s = fs[i];
                    own[s] = mine;
                } else if (own[fs[i]] == ORC_DRAIN) {
                    own[s] = ORC_EMPTY;
                    removed = true;
                }
            }
            if (!removed) site[w++] = s;
        }
        return w;
    };
    ne = tick(e_site, ef.data(), ne, et, ORC_ELECTRON, e_rm);
    nh = tick(h_site, hf.data(), nh, ht, ORC_HOLE, h_rm);

    // SourceAgent::tryToInject for electrode source s (0 eL, 1 eR, 2 hL, 3 hR)
    // on the draw at {step, index, purpose} (sourceagent.cpp:92-103): the site
    // from the face (randomNeighborSiteID over the sorted face slice,
    // cubicgrid.cpp:167-205, 473-487), validToInject (sourceagent.cpp:192-232),
    // then shouldTransport (sourceagent.cpp:168-181): chooseYes on the rate,
    // or with source.metropolis the Metropolis test on energyChange
    // (sourceagent.cpp:125-161; the source's own potential is 0, never set).
    const double src_rate[4] = {k->rate_e_source_l, k->rate_e_source_r, k->rate_h_source_l,
                                k->rate_h_source_r};
    std::vector<uint8_t> is_defect(V, 0);
    for (int i = 0; i < nd; ++i) is_defect[defects[i]] = 1;
    auto try_inject = [&](int s, uint32_t index, uint32_t purpose) {
        const bool electron = s < 2;
        const bool left = (s % 2) == 0;
        counters[2 * s] += 1;  // attempts (sourceagent.cpp:94)
        const Draw d = draw(k, step, index, purpose);
        const uint32_t idx = uint_below(d.w[0], (uint32_t)(GY * GZ));
        const int site = GX * (int)idx + (left ? 0 : GX - 1);
        std::vector<uint8_t>& own = electron ? et : ht;
        const int count = electron ? ne : nh;
        const int cap = electron ? k->max_electrons : k->max_holes;
        const bool valid =
            count < cap && src_rate[s] > 0 && own[site] == ORC_EMPTY && !is_defect[site];
        if (!valid) return;
        const double u = unit_double(d.w[1], d.w[2]);
        bool accept;
        if (k->source_metropolis) {
            double p2 = pot[site];
            if (k->source_coulomb) {
                // p2 += coulombH + coulombImageH + coulombE + coulombImageE
                // (+ coulombD + coulombImageD), point charges, in that order
                std::vector<int32_t> qh(nh, 1), qe(ne, -1), qd(nd, k->defects_charge);
                p2 += orc_species_potential(ctx, site, h_site, qh.data(), nh, 0, 0);
                p2 += orc_species_potential(ctx, site, h_site, qh.data(), nh, 0, 1);
                p2 += orc_species_potential(ctx, site, e_site, qe.data(), ne, 0, 0);
                p2 += orc_species_potential(ctx, site, e_site, qe.data(), ne, 0, 1);
                if (k->defects_charge != 0) {
                    p2 += orc_species_potential(ctx, site, defects, qd.data(), nd, 0, 0);
                    p2 += orc_species_potential(ctx, site, defects, qd.data(), nd, 0, 1);
                }
            }
            const double de = electron ? 0.0 - p2 : p2 - 0.0;
            // Random::metropolisWithCoupling (rand.cpp:91-106), coupling = rate
            accept = de > 0.0 ? src_rate[s] * std::exp(-de * k->inverse_kt) > u : src_rate[s] > u;
        } else {
            accept = src_rate[s] > u;  // chooseYes (rand.cpp:117-124)
        }
        if (accept) {
            counters[2 * s + 1] += 1;
            own[site] = electron ? ORC_ELECTRON : ORC_HOLE;
            if (electron) e_site[ne++] = site;
            else h_site[nh++] = site;
        }
    };

    if (k->solar) {
        // performInjections, solar (simulation.cpp:235-243): the exciton source,
        // ExcitonSourceAgent::tryToInject (sourceagent.cpp:92-103, 120-123, 234-250).
        counters[16] += 1;
        const Draw d = draw(k, step, 0u, 20u);
        int es, hs;
        if (k->bonds && k->nbonds > 0) {
            const uint32_t b = uint_below(d.w[0], (uint32_t)k->nbonds);
            hs = k->bonds[2 * b];
            es = k->bonds[2 * b + 1];
        } else {
            es = hs = (int)uint_below(d.w[0], (uint32_t)V);
        }
        const bool valid = ne < k->max_electrons && nh < k->max_holes &&
                           k->generation_rate > 0 && et[es] == ORC_EMPTY && ht[hs] == ORC_EMPTY &&
                           (k->bonds && k->nbonds > 0 ? true : ht[es] == ORC_EMPTY);
        if (valid && k->generation_rate > unit_double(d.w[1], d.w[2])) {
            counters[17] += 1;
            et[es] = ORC_ELECTRON;
            ht[hs] = ORC_HOLE;
            e_site[ne++] = es;
            h_site[nh++] = hs;
        }
        // Simulation::balanceCharges (simulation.cpp:253-353): electrons from
        // the electrode on the low-potential side (a uniform draw picks it when
        // the voltages are equal) until electrons >= holes, then holes alike;
        // try t of a species draws at {step, t, 24 / 26} (25 / 27: the side)
        if (k->balance_charges) {
            for (int species = 0; species < 2; ++species) {
                const bool electron = species == 0;
                for (int t = 0;; ++t) {
                    const int more = electron ? nh - ne : ne - nh;
                    const bool at_max = electron ? ne >= k->max_electrons : nh >= k->max_holes;
                    if (more <= 0 || at_max) break;
                    if (t >= 1024) return -1;  // qFatal "can not balance ..."
                    bool left;
                    if (k->voltage_right > k->voltage_left) left = electron;
                    else if (k->voltage_left > k->voltage_right) left = !electron;
                    else {
                        const Draw d = draw(k, step, (uint32_t)t, electron ? 25u : 27u);
                        const bool above = unit_double(d.w[0], d.w[1]) > 0.5;
                        left = electron ? above : !above;
                    }
                    try_inject((electron ? 0 : 2) + (left ? 0 : 1), (uint32_t)t,
                               electron ? 24u : 26u);
                }
            }
        }
        *ne_io = ne;
        *nh_io = nh;
        return 0;
    }

    // performInjections, transistor (simulation.cpp:246-249): eL, eR, hL, hR.
    for (int s = 0; s < 4; ++s) try_inject(s, 0u, 16u + (uint32_t)s);
    *ne_io = ne;
    *nh_io = nh;
    return 0;
}
