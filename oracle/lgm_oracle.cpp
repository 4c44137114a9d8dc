// lgm_oracle.cpp -- CPU FP64 oracle for the Coulomb hot path (TEST INFRASTRUCTURE).
//
// Restates the reference engine's CPU Coulomb path and the semantics of its
// OpenCL kernels in plain C++.  Not part of the product: see lgm_oracle.h for
// who may load it and for the pins that tie it to the reference.
#include "lgm_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

struct orc_ctx {
    int X, Y, Z;            // grid.x, grid.y, grid.z
    int XY, volume;
    int cutoff;             // electrostatic.cutoff
    int hopping_range;      // hopping.range
    double sigma;           // coulomb.gaussian.sigma
    double prefactor;       // electrostatic.prefactor
    int n;                  // cutoff + 1 (table edge)
    int nh;                 // hopping_range + 1
    std::vector<double> R1, R2, iR, eR, sI, coupling;
};

namespace {

inline int tix(const orc_ctx* c, int dx, int dy, int dz) {
    return (dx * c->n + dy) * c->n + dz;
}

inline int hix(const orc_ctx* c, int dx, int dy, int dz) {
    return (dx * c->nh + dy) * c->nh + dz;
}

// Grid::getIndexX/Y/Z (cubicgrid.cpp:132-145)
inline int gx(const orc_ctx* c, int s) { return s % c->X; }
inline int gy(const orc_ctx* c, int s) { return s / c->X - (s / c->XY) * c->Y; }
inline int gz(const orc_ctx* c, int s) { return s / c->XY; }

template <class F>
void parallel_for(int n, int threads, F&& body) {
    if (threads <= 0) {
        threads = (int)std::thread::hardware_concurrency();
        if (threads <= 0) threads = 1;
    }
    if (threads == 1 || n < 2) {
        for (int i = 0; i < n; ++i) body(i);
        return;
    }
    std::atomic<int> next(0);
    const int grain = std::max(1, n / (threads * 16));
    auto worker = [&]() {
        for (;;) {
            int b = next.fetch_add(grain);
            if (b >= n) break;
            int e = std::min(n, b + grain);
            for (int i = b; i < e; ++i) body(i);
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(threads - 1);
    for (int t = 0; t < threads - 1; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// Potential::coulombE/H/D, gaussE/H/D and their Image variants
// (potential.cpp:351-753).  One loop shape serves all twelve: the species
// list, the distance function (direct or x-image) and the eR factor differ.
// `mirror` selects the x distance: 0 direct |x_i - x_j| (cubicgrid.cpp:102-105),
// 1 left image x_i + x_j + 1 (cubicgrid.cpp:117-120), 2 right image
// (2X - 1 - x_i - x_j, an extension with the same cutoff rules).
double species_sum(const orc_ctx* c, int site_i, const int32_t* sites,
                   const int32_t* charges, int n, bool gauss, int mirror) {
    const int cutoff = c->cutoff;
    const int xi = gx(c, site_i), yi = gy(c, site_i), zi = gz(c, site_i);
    double potential = 0.0;
    for (int j = 0; j < n; ++j) {
        const int site_j = sites[j];
        const int xj = gx(c, site_j), yj = gy(c, site_j), zj = gz(c, site_j);
        int dx;
        if (mirror == 0) dx = std::abs(xi - xj);
        else if (mirror == 1) dx = std::abs(xi + xj) + 1;
        else dx = std::abs(2 * c->X - 1 - xi - xj);
        const int dy = std::abs(yi - yj);
        const int dz = std::abs(zi - zj);
        if ((dx < cutoff) && (dy < cutoff) && (dz < cutoff)) {
            const int t = tix(c, dx, dy, dz);
            if (c->R1[t] < cutoff) {
                double term = gauss ? (c->iR[t] * charges[j] * c->eR[t])
                                    : (c->iR[t] * charges[j]);
                if (mirror == 0) potential += term;
                else potential -= term;
            }
        }
    }
    return potential * c->prefactor;
}

}  // namespace

extern "C" {

// World::initialize (world.cpp:589-647): grids, then precalculateArrays
// (potential.cpp:246-324) and updateCouplingConstants (potential.cpp:326-349).
orc_ctx* orc_create(int grid_x, int grid_y, int grid_z, int cutoff,
                    int hopping_range, double sigma, double prefactor) {
    if (grid_x < 1 || grid_y < 1 || grid_z < 1 || cutoff < 1 ||
        hopping_range < 1 || hopping_range > 2)
        return nullptr;
    orc_ctx* c = new orc_ctx();
    c->X = grid_x; c->Y = grid_y; c->Z = grid_z;
    c->XY = grid_x * grid_y;
    c->volume = c->XY * grid_z;
    c->cutoff = cutoff;
    c->hopping_range = hopping_range;
    c->sigma = sigma;
    c->prefactor = prefactor;
    c->n = cutoff + 1;
    c->nh = hopping_range + 1;
    const size_t n3 = (size_t)c->n * c->n * c->n;
    c->R1.assign(n3, 0.0); c->R2.assign(n3, 0.0);
    c->iR.assign(n3, 0.0); c->eR.assign(n3, 1.0);
    // potential.cpp:268-290
    for (int dx = 0; dx < c->n; ++dx)
        for (int dy = 0; dy < c->n; ++dy)
            for (int dz = 0; dz < c->n; ++dz) {
                double r2 = dx * dx + dy * dy + dz * dz;
                double r1 = 0.0, ir = 0.0;
                if (r2 > 0) { r1 = std::sqrt(r2); ir = 1.0 / r1; }
                const int t = tix(c, dx, dy, dz);
                c->R2[t] = r2; c->R1[t] = r1; c->iR[t] = ir; c->eR[t] = 1.0;
            }
    // potential.cpp:293-308
    if (sigma > 0.0) {
        const double factor = 1.0 / (std::sqrt(2.0) * sigma);
        for (size_t t = 0; t < n3; ++t) c->eR[t] = std::erf(factor * c->R1[t]);
    }
    // potential.cpp:311-323 (sI needs (h+1) <= (cutoff+1))
    const size_t h3 = (size_t)c->nh * c->nh * c->nh;
    c->sI.assign(h3, 0.0);
    for (int dx = 0; dx < c->nh; ++dx)
        for (int dy = 0; dy < c->nh; ++dy)
            for (int dz = 0; dz < c->nh; ++dz) {
                const int t = tix(c, dx, dy, dz);
                c->sI[hix(c, dx, dy, dz)] = prefactor * c->iR[t] * c->eR[t];
            }
    // potential.cpp:326-349
    c->coupling.assign(h3, 0.0);
    const double c1 = 1.0 / 3.0, c2 = 1.0 / 27.0;
    for (int dx = 0; dx < c->nh; ++dx)
        for (int dy = 0; dy < c->nh; ++dy)
            for (int dz = 0; dz < c->nh; ++dz) {
                double r = std::sqrt((double)(dx * dx + dy * dy + dz * dz));
                c->coupling[hix(c, dx, dy, dz)] =
                    c1 * std::pow(3.0, r - 1) * std::pow(c2, r - 1);
            }
    c->coupling[0] = 0.0;
    return c;
}

void orc_destroy(orc_ctx* ctx) { delete ctx; }

void orc_table(const orc_ctx* c, int which, double* out) {
    const std::vector<double>* v = which == 0 ? &c->R1 : which == 1 ? &c->R2
                                 : which == 2 ? &c->iR : &c->eR;
    std::memcpy(out, v->data(), v->size() * sizeof(double));
}

void orc_self_table(const orc_ctx* c, double* out) {
    std::memcpy(out, c->sI.data(), c->sI.size() * sizeof(double));
}

void orc_coupling_table(const orc_ctx* c, double* out) {
    std::memcpy(out, c->coupling.data(), c->coupling.size() * sizeof(double));
}

void orc_dims(const orc_ctx* c, int dims[3]) { dims[0] = c->X; dims[1] = c->Y; dims[2] = c->Z; }
int orc_hopping_range(const orc_ctx* c) { return c->hopping_range; }
double orc_sigma(const orc_ctx* c) { return c->sigma; }

int orc_index_x(const orc_ctx* c, int s) { return gx(c, s); }
int orc_index_y(const orc_ctx* c, int s) { return gy(c, s); }
int orc_index_z(const orc_ctx* c, int s) { return gz(c, s); }
// Grid::getIndexS (cubicgrid.cpp:162-165)
int orc_index_s(const orc_ctx* c, int x, int y, int z) { return c->X * (y + z * c->Y) + x; }

// Grid::neighborsSite (cubicgrid.cpp:207-446), lattice part only, in the
// reference's push order (the order fixes which id a uniform draw selects).
int orc_neighbors(const orc_ctx* c, int site, int hr, int* out) {
    const int x = gx(c, site), y = gy(c, site), z = gz(c, site);
    const int X = c->X, Y = c->Y, Z = c->Z;
    int n = 0;
    auto S = [&](int a, int b, int d) { out[n++] = orc_index_s(c, a, b, d); };
    if (hr == 1) {
        if (x > 0) S(x - 1, y, z);
        if (x < X - 1) S(x + 1, y, z);
        if (y > 0) S(x, y - 1, z);
        if (y < Y - 1) S(x, y + 1, z);
        if (z > 0) S(x, y, z - 1);
        if (z < Z - 1) S(x, y, z + 1);
    } else if (hr == 2) {
        if (Z == 1) {
            if (x > 0) {
                S(x - 1, y, z);
                if (y > 0) S(x - 1, y - 1, z);
                if (y < Y - 1) S(x - 1, y + 1, z);
                if (x > 1) S(x - 2, y, z);
            }
            if (x < X - 1) {
                S(x + 1, y, z);
                if (y > 0) S(x + 1, y - 1, z);
                if (y < Y - 1) S(x + 1, y + 1, z);
                if (x < X - 2) S(x + 2, y, z);
            }
            if (y > 0) {
                S(x, y - 1, z);
                if (y > 1) S(x, y - 2, z);
            }
            if (y < Y - 1) {
                S(x, y + 1, z);
                if (y < Y - 2) S(x, y + 2, z);
            }
        } else {
            if (x > 0) {
                S(x - 1, y, z);
                if (y > 0) {
                    S(x - 1, y - 1, z);
                    if (z > 0) S(x - 1, y - 1, z - 1);
                    if (z < Z - 1) S(x - 1, y - 1, z + 1);
                }
                if (y < Y - 1) {
                    S(x - 1, y + 1, z);
                    if (z > 0) S(x - 1, y + 1, z - 1);
                    if (z < Z - 1) S(x - 1, y + 1, z + 1);
                }
                if (z > 0) S(x - 1, y, z - 1);
                if (z < Z - 1) S(x - 1, y, z + 1);
                if (x > 1) S(x - 2, y, z);
            }
            if (x < X - 1) {
                S(x + 1, y, z);
                if (y > 0) {
                    S(x + 1, y - 1, z);
                    if (z > 0) S(x + 1, y - 1, z - 1);
                    if (z < Z - 1) S(x + 1, y - 1, z + 1);
                }
                if (y < Y - 1) {
                    S(x + 1, y + 1, z);
                    if (z > 0) S(x + 1, y + 1, z - 1);
                    if (z < Z - 1) S(x + 1, y + 1, z + 1);
                }
                if (z > 0) S(x + 1, y, z - 1);
                if (z < Z - 1) S(x + 1, y, z + 1);
                if (x < X - 2) S(x + 2, y, z);
            }
            if (z > 0) {
                S(x, y, z - 1);
                if (y > 0) S(x, y - 1, z - 1);
                if (y < Y - 1) S(x, y + 1, z - 1);
                if (z > 1) S(x, y, z - 2);
            }
            if (z < Z - 1) {
                S(x, y, z + 1);
                if (y > 0) S(x, y - 1, z + 1);
                if (y < Y - 1) S(x, y + 1, z + 1);
                if (z < Z - 2) S(x, y, z + 2);
            }
            if (y > 0) {
                S(x, y - 1, z);
                if (y > 1) S(x, y - 2, z);
            }
            if (y < Y - 1) {
                S(x, y + 1, z);
                if (y < Y - 2) S(x, y + 2, z);
            }
        }
    }
    return n;
}

double orc_species_potential(const orc_ctx* c, int site_i, const int32_t* sites,
                             const int32_t* charges, int n, int gauss, int image) {
    return species_sum(c, site_i, sites, charges, n, gauss != 0, image ? 1 : 0);
}

double orc_species_potential_right_image(const orc_ctx* c, int site_i,
                                         const int32_t* sites, const int32_t* charges,
                                         int n, int gauss) {
    return species_sum(c, site_i, sites, charges, n, gauss != 0, 2);
}

void orc_potentials(const orc_ctx* c, int gauss, unsigned terms, const int32_t* src,
                    const int32_t* q, int n, const int32_t* tgt, int t, double* out,
                    int threads) {
    parallel_for(t, threads, [&](int g) {
        double v = 0.0;
        if (terms & 1u) v += species_sum(c, tgt[g], src, q, n, gauss != 0, 0);
        if (terms & 2u) v += species_sum(c, tgt[g], src, q, n, gauss != 0, 1);
        if (terms & 4u) v += species_sum(c, tgt[g], src, q, n, gauss != 0, 2);
        out[g] = v;
    });
}

// coulomb2 / gauss2 (kernel.cl:222-369): decode (x,y,z) from the site id with
// xsize/ysize (kernel.cl:229-231, 266-268), integer r^2, keep 0 < r2 < c2,
// accumulate q*rsqrt(r2) or q*erf(f*r)/r, scale by prefactor.
void orc_kernel2(const orc_ctx* c, int kind, const int32_t* s, const int32_t* q,
                 int n, int total, double* o, int threads) {
    const int c2 = c->cutoff * c->cutoff;
    const int X = c->X, XY = c->XY, Y = c->Y;
    const double erffactor = c->sigma > 0 ? 1.0 / (std::sqrt(2.0) * c->sigma) : 0.0;
    std::vector<int> xs(n), ys(n), zs(n);
    for (int j = 0; j < n; ++j) {
        const int sj = s[j];
        zs[j] = sj / XY; ys[j] = sj / X - zs[j] * Y; xs[j] = sj % X;
    }
    parallel_for(total, threads, [&](int g) {
        const int si = s[g];
        const int zi = si / XY, yi = si / X - zi * Y, xi = si % X;
        double v = 0.0;
        for (int j = 0; j < n; ++j) {
            const int dx = xi - xs[j], dy = yi - ys[j], dz = zi - zs[j];
            const double r = dx * dx + dy * dy + dz * dz;
            if (r > 0 && r < c2) {
                if (kind == 0) {
                    v += q[j] * (1.0 / std::sqrt(r));
                } else {
                    const double rr = std::sqrt(r);
                    v += q[j] * std::erf(erffactor * rr) / rr;
                }
            }
        }
        o[g] = c->prefactor * v;
    });
}

// coulomb1 / gauss1 (kernel.cl:56-220): one value per lattice site k, the
// site's (x,y,z) being its work-group id, charges decoded with the group
// counts (= grid dims).
void orc_kernel1(const orc_ctx* c, int kind, const int32_t* s, const int32_t* q,
                 int n, double* o, int threads) {
    const int c2 = c->cutoff * c->cutoff;
    const int X = c->X, XY = c->XY, Y = c->Y;
    const double erffactor = c->sigma > 0 ? 1.0 / (std::sqrt(2.0) * c->sigma) : 0.0;
    std::vector<int> xs(n), ys(n), zs(n);
    for (int j = 0; j < n; ++j) {
        const int sj = s[j];
        zs[j] = sj / XY; ys[j] = sj / X - zs[j] * Y; xs[j] = sj % X;
    }
    parallel_for(c->volume, threads, [&](int k) {
        const int xi = k % X, yi = (k / X) % Y, zi = k / XY;
        double v = 0.0;
        for (int j = 0; j < n; ++j) {
            const int dx = xi - xs[j], dy = yi - ys[j], dz = zi - zs[j];
            const double r = dx * dx + dy * dy + dz * dz;
            if (r > 0 && r < c2) {
                if (kind == 0) {
                    v += q[j] * (1.0 / std::sqrt(r));
                } else {
                    const double rr = std::sqrt(r);
                    v += q[j] * std::erf(erffactor * rr) / rr;
                }
            }
        }
        o[k] = c->prefactor * v;
    });
}

// ChargeAgent::coulombCPU (chargeagent.cpp:215-271) for every carrier, with
// bindingPotential (chargeagent.cpp:463-481).  Species order of the sums and
// the per-species calls follow the reference; defect sums only when
// defects.charge != 0 (chargeagent.cpp:238, 256).
void orc_coulomb_cpu(const orc_ctx* c,
                     const int32_t* e_site, const int32_t* e_fsite, int ne,
                     const int32_t* h_site, const int32_t* h_fsite, int nh,
                     const int32_t* d_site, int nd, int defects_charge,
                     const uint8_t* e_type, const uint8_t* h_type,
                     double exciton_binding,
                     double* de_out, double* p1_out, double* p2_out,
                     int threads) {
    std::vector<int32_t> eq(ne, -1), hq(nh, +1), dq(nd, defects_charge);
    const bool gauss = c->sigma > 0;
    const double sI100 = c->sI[hix(c, 1, 0, 0)];
    parallel_for(ne + nh, threads, [&](int i) {
        const bool is_e = i < ne;
        const int k = is_e ? i : i - ne;
        const int site = is_e ? e_site[k] : h_site[k];
        const int fsite = is_e ? e_fsite[k] : h_fsite[k];
        const int charge = is_e ? -1 : +1;
        double p1 = 0, p2 = 0;
        const double self = sI100 * charge;
        // Electrons, holes, charged defects (chargeagent.cpp:227-261)
        p1 += species_sum(c, site, e_site, eq.data(), ne, gauss, 0);
        p2 += species_sum(c, fsite, e_site, eq.data(), ne, gauss, 0);
        p1 += species_sum(c, site, h_site, hq.data(), nh, gauss, 0);
        p2 += species_sum(c, fsite, h_site, hq.data(), nh, gauss, 0);
        if (defects_charge != 0) {
            p1 += species_sum(c, site, d_site, dq.data(), nd, gauss, 0);
            p2 += species_sum(c, fsite, d_site, dq.data(), nd, gauss, 0);
        }
        p2 -= self;  // chargeagent.cpp:264
        // bindingPotential (chargeagent.cpp:463-481)
        auto bind = [&](int st) -> double {
            if (is_e) return h_type[st] == ORC_HOLE ? sI100 + exciton_binding : 0.0;
            return e_type[st] == ORC_ELECTRON ? sI100 - exciton_binding : 0.0;
        };
        p2 += bind(fsite);
        p1 += bind(site);
        de_out[i] = charge * (p2 - p1);
        if (p1_out) p1_out[i] = p1;
        if (p2_out) p2_out[i] = p2;
    });
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the
// published multipliers and Weyl key increments.
void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

}  // extern "C"
